"""Numpy restatement of the reference integrator, vectorised over runs.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Each run is one lane of a batch; control flow that the reference executes
per CUDA thread becomes a boolean mask per run.  Arithmetic runs in the
system precision (``float32`` or ``float64``), as the reference's device
code does; with ``control_dtype=float64`` time, step size, controller and
norms run in float64 and the state update is compensated, which is the
engine's mixed-precision mode.

Followed files (reference, ``src/cubie/``):
  loop             integrators/loops/ode_loop.py:493-984
  schedules        integrators/SingleIntegratorRun.py:153-292
  ERK step         integrators/algorithms/generic_erk.py:359-577
  Rosenbrock step  integrators/algorithms/generic_rosenbrock_w.py:459-759
  FIRK step        integrators/algorithms/generic_firk.py:508-701
  DIRK step        integrators/algorithms/generic_dirk.py:515-855
  mass matrix      odesystems/symbolic/codegen/linear_operators.py:708-735,
                   nonlinear_residuals.py:59-130,324-345 (M v and M u terms;
                   Rosenbrock's C_ij k_j / h term with M applied, where the
                   reference, generic_rosenbrock_w.py:682-698, omits it)
  dense predictor  integrators/stage_predictors.py:76-548
  Newton           integrators/matrix_free_solvers/newton_krylov.py:340-517
  MR / SD          integrators/matrix_free_solvers/linear_solver.py:220-385
  BiCGSTAB         integrators/matrix_free_solvers/bicgstab_solver.py:367-663
  norms            integrators/norms.py:165-435
  controllers      integrators/step_control/adaptive_{I,PI,PID}_controller.py,
                   gustafsson_controller.py
  summaries        outputhandling/summarymetrics/{mean,max,min,rms,std,extrema,peaks}.py
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np
import sympy as sp

# ---------------------------------------------------------------------------
# Tableaus (published coefficients, as tabulated by the reference)
# ---------------------------------------------------------------------------


@dataclass
class OTab:
    kind: str
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    order: int
    b_hat: Optional[np.ndarray] = None
    C: Optional[np.ndarray] = None
    gamma: float = 0.0
    gamma_stages: Optional[np.ndarray] = None
    dense32: float = 0.0
    dense64: float = 0.0
    # DIRK: an implicit stage after an explicit one starts Newton from h
    # times that stage's derivative (explicit Euler predictor)
    euler_guess: bool = False

    @property
    def s(self):
        return len(self.b)

    @property
    def d(self):
        return None if self.b_hat is None else self.b - self.b_hat

    @property
    def has_err(self):
        return self.b_hat is not None and np.any(self.b - self.b_hat != 0.0)

    def row_match(self, w):
        if w is None:
            return None
        m = None
        for r in range(self.s):
            if np.all(np.abs(self.a[r] - w) <= 1e-15):
                m = r
        return m


def _tab(kind, a, b, c, order, **kw):
    s = len(b)
    A = np.zeros((s, s))
    for i, row in enumerate(a):
        A[i, :len(row)] = row
    out = OTab(kind, A, np.array(b, float), np.array(c, float), order, **kw)
    if out.b_hat is not None:
        out.b_hat = np.array(out.b_hat, float)
    return out


def _ros3p():
    g = 0.5 + math.sqrt(3.0) / 6.0
    ig = 1.0 / g
    b_aux = ig * (2.0 / 3.0 - ig / 6.0)
    C = np.array([[0, 0, 0], [-(ig ** 2), 0, 0],
                  [-ig * (1.0 + ig * (2.0 - 0.5 * ig)), -ig * (2.0 - 0.5 * ig), 0]])
    return _tab("rosenbrock", [[0, 0, 0], [ig, 0, 0], [ig, 0, 0]],
                [ig * (1.0 + b_aux), b_aux, ig / 3.0], [0, 1, 1], 3,
                b_hat=[2.113248654051871, 1.0, 0.4226497308103742], C=C, gamma=g,
                gamma_stages=np.array([g, -0.2113248654051871, 0.5 - 2.0 * g]))


def _radau():
    s6 = math.sqrt(6.0)
    c = np.array([(4 - s6) / 10.0, (4 + s6) / 10.0, 1.0])
    M = np.vander(c, N=2, increasing=True).T
    bh = np.linalg.lstsq(M, np.array([1.0, 0.5]), rcond=None)[0]
    a = [[(88 - 7 * s6) / 360.0, (296 - 169 * s6) / 1800.0, (-2 + 3 * s6) / 225.0],
         [(296 + 169 * s6) / 1800.0, (88 + 7 * s6) / 360.0, (-2 - 3 * s6) / 225.0],
         [(16 - s6) / 36.0, (16 + s6) / 36.0, 1.0 / 9.0]]
    return _tab("firk", a, a[2], c, 5, b_hat=bh, dense32=8.0, dense64=8.0)


def _dirk3():
    s2, s6 = math.sqrt(2.0), math.sqrt(6.0)
    arc = math.atan(s2 / 4.0) / 3.0
    g = -s2 * math.cos(arc) / 2.0 + s6 * math.sin(arc) / 2.0 + 1.0
    b1 = (-6.0 * g ** 2 + 16.0 * g - 1.0) / 4.0
    b2 = (6.0 * g ** 2 - 20.0 * g + 5.0) / 4.0
    return _tab("dirk", [[g], [(1.0 - g) / 2.0, g], [b1, b2, g]], [b1, b2, g], [g, (1.0 + g) / 2.0, 1.0], 3,
                dense32=0.85, dense64=1.07)


TABLEAUS: Dict[str, OTab] = {
    "dormand-prince-54": _tab(
        "erk",
        [[0], [1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9],
         [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
         [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
         [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]],
        [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0],
        [0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1, 1], 5,
        b_hat=[5179 / 57600, 0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]),
    "classical-rk4": _tab("erk", [[0], [0.5], [0, 0.5], [0, 0, 1]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0, .5, .5, 1], 4),
    "ros3p": _ros3p(),
    "radau_iia_5": _radau(),
    "l_stable_dirk_3": _dirk3(),
    "l_stable_sdirk_4": _tab(
        "dirk",
        [[0.25], [0.5, 0.25], [17 / 50, -1 / 25, 0.25], [371 / 1360, -137 / 2720, 15 / 544, 0.25],
         [25 / 24, -49 / 48, 125 / 16, -85 / 12, 0.25]],
        [25 / 24, -49 / 48, 125 / 16, -85 / 12, 0.25], [0.25, 0.75, 11 / 20, 0.5, 1.0], 4,
        b_hat=[59 / 48, -17 / 96, 225 / 32, -85 / 12, 0.0], dense32=0.79, dense64=0.79),
}
TABLEAUS["radau"] = TABLEAUS["radau_iia_5"]
TABLEAUS["rk45"] = TABLEAUS["dormand-prince-54"]

# The reference's single-purpose steps, restated as tableaus:
#   explicit Euler (explicit_euler.py: y + h f(t, y));
#   backward Euler (backwards_euler.py: z = h f(t + h, y + z), Newton seeded
#   with the previous step's increment);
#   backward Euler with an explicit Euler predictor
#   (backwards_euler_predict_correct.py: Newton seeded with h f(t, y));
#   Crank-Nicolson (crank_nicolson.py: trapezoidal solve seeded with h f(t, y),
#   then a backward Euler solve seeded with the trapezoidal increment; the
#   error is their difference).
TABLEAUS["euler"] = _tab("erk", [[0]], [1.0], [0.0], 1)
TABLEAUS["backwards_euler"] = _tab("dirk", [[1.0]], [1.0], [1.0], 1)
TABLEAUS["backwards_euler_pc"] = _tab("dirk", [[0, 0], [0, 1.0]], [0.0, 1.0], [0.0, 1.0], 1, euler_guess=True)
TABLEAUS["crank_nicolson"] = _tab("dirk", [[0, 0, 0], [0.5, 0.5, 0], [0, 0, 1.0]], [0.5, 0.5, 0.0],
                                  [0.0, 1.0, 1.0], 2, b_hat=[0.0, 0.0, 1.0], euler_guess=True)


def load_reference_tableaus(path) -> int:
    """Add every tableau of a coefficient file written from the reference's
    registries (``tests/golden/make_tableau_fixture.py``: ``<alias>/a``,
    ``/b``, ``/c``, ``/b_hat``, ``/C``, ...) whose alias is not restated
    above; returns the number added."""
    data = np.load(path)
    aliases = sorted({k.split("/")[0] for k in data.files})
    added = 0
    for al in aliases:
        if al in TABLEAUS:
            continue
        g = lambda f: data[f"{al}/{f}"] if f"{al}/{f}" in data.files else None
        kind = str(g("kind"))
        kw = dict(dense32=float(g("dense32")), dense64=float(g("dense64")))
        if g("b_hat") is not None:
            kw["b_hat"] = g("b_hat")
        if kind == "rosenbrock":
            kw.update(C=g("C"), gamma=float(g("gamma")), gamma_stages=g("gamma_stages"))
        TABLEAUS[al] = _tab(kind, g("a"), g("b"), g("c"), int(g("order")), **kw)
        added += 1
    return added


_REFERENCE_TABLEAUS = Path(__file__).resolve().parent.parent / "tests" / "golden" / "ref_tableaus.npz"
if _REFERENCE_TABLEAUS.exists():
    load_reference_tableaus(_REFERENCE_TABLEAUS)

FAMILY_CONTROLLER = {
    "erk": dict(step_controller="pi", kp=0.7, ki=-0.4, deadband_min=1.0, deadband_max=1.0,
                min_gain=0.2, max_gain=10.0, safety=0.9),
    "rosenbrock": dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
                       min_gain=0.2, max_gain=8.0, safety=0.9),
    "firk": dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
                 min_gain=0.2, max_gain=8.0, safety=0.9),
    "dirk": dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
                 min_gain=0.2, max_gain=8.0, safety=0.9),
}


def _pred_coeffs(tab: OTab) -> np.ndarray:
    """Dense read-ahead polynomial coefficients [power, target, source]."""
    nodes = tab.c
    last = {}
    for st, nd in enumerate(nodes):
        last[nd] = st
    samples = list(last.values())
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
        cf[:len(poly.coef)] = poly.coef
        shifted.append(cf)
    out = np.zeros((k, tab.s, tab.s))
    for p in range(k):
        for t in range(tab.s):
            for bi in range(k):
                out[p, t, samples[bi]] = shifted[bi][p] * nodes[t] ** p
    return out


# ---------------------------------------------------------------------------
# System
# ---------------------------------------------------------------------------
class OracleSystem:
    """``dy/dt = f(t, y, p)`` from ``lhs = rhs`` strings, evaluated by
    SymPy-generated numpy functions over a batch of runs."""

    def __init__(self, equations: Sequence[str], states: Sequence[str], parameters: Sequence[str] = (),
                 constants: Optional[Dict[str, float]] = None, observables: Sequence[str] = (),
                 drivers: Sequence[str] = (), mass=None):
        constants = constants or {}
        # constant mass matrix of M y' = f (None: identity), as the
        # reference's create_ODE_system ``mass`` (symbolicODE.py:179-184)
        self.mass = None if mass is None else np.asarray(mass, dtype=np.float64)
        self.states = list(states)
        self.parameters = list(parameters)
        self.observables = list(observables)
        self.drivers = list(drivers)
        self.driver_table: Optional["DriverTable"] = None
        t = sp.Symbol("t", real=True)
        table = {nm: sp.Symbol(nm, real=True) for nm in self.states + self.parameters + self.drivers}
        table.update({k: sp.Float(v, 17) for k, v in constants.items()})
        table["t"] = t
        aux = {}
        derivs = {}
        for eq in equations:
            lhs, rhs = [x.strip() for x in eq.split("=", 1)]
            expr = sp.sympify(rhs, locals={**table, **aux})
            expr = expr.xreplace(aux)
            if lhs.startswith("d") and lhs[1:] in self.states:
                derivs[lhs[1:]] = expr
                aux[sp.Symbol(lhs, real=True)] = expr
                table[lhs] = expr
            else:
                aux[sp.Symbol(lhs, real=True)] = expr
                table[lhs] = expr
        self.n = len(self.states)
        ys = [table[s] for s in self.states]
        ps = [table[p] for p in self.parameters]
        ds = [table[d] for d in self.drivers]
        dds = [sp.Symbol(f"_ddot_{d}", real=True) for d in self.drivers]
        f = [derivs[s] for s in self.states]
        J = sp.Matrix(f).jacobian(sp.Matrix(ys))
        args = (t, ys, ps, ds)
        self._f = sp.lambdify(args, f, "numpy")
        self._J = sp.lambdify(args, J.tolist(), "numpy")
        # time derivative with the driver chain rule (time_derivative.py:51)
        dfdt = [sp.diff(e, t) + sum((sp.diff(e, d) * dd for d, dd in zip(ds, dds)), sp.Integer(0)) for e in f]
        self._dt = sp.lambdify((t, ys, ps, ds, dds), dfdt, "numpy")
        self._obs = sp.lambdify(args, [table[o] for o in self.observables], "numpy") if self.observables else None

    def mv(self, v: np.ndarray) -> np.ndarray:
        """M v for every run (rows of ``v``); v itself without a mass matrix."""
        if self.mass is None:
            return v
        return (v @ self.mass.T.astype(v.dtype)).astype(v.dtype)

    def _drv(self, t, B, dtype, derivative=False):
        """Driver values (or time derivatives) at ``t`` for every run."""
        if not self.drivers:
            return []
        if self.driver_table is None:
            raise ValueError("the system has drivers: set ``driver_table`` first")
        tt = np.broadcast_to(np.asarray(t, dtype=dtype), (B,))
        vals = self.driver_table.evaluate(tt, derivative)
        return [vals[:, k] for k in range(vals.shape[1])]

    @staticmethod
    def _stack(vals, B, dtype):
        return np.stack([np.broadcast_to(np.asarray(v, dtype=dtype), (B,)) for v in vals], axis=-1)

    def f(self, t, Y, P):
        B = Y.shape[0]
        dtype = Y.dtype
        return self._stack(self._f(t, [Y[:, i] for i in range(self.n)], [P[:, j] for j in range(P.shape[1])],
                                   self._drv(t, B, dtype)), B, dtype)

    def jac(self, t, Y, P):
        B = Y.shape[0]
        dtype = Y.dtype
        rows = self._J(t, [Y[:, i] for i in range(self.n)], [P[:, j] for j in range(P.shape[1])],
                       self._drv(t, B, dtype))
        return np.stack([self._stack(r, B, dtype) for r in rows], axis=1)

    def dfdt(self, t, Y, P):
        B = Y.shape[0]
        return self._stack(self._dt(t, [Y[:, i] for i in range(self.n)], [P[:, j] for j in range(P.shape[1])],
                                    self._drv(t, B, Y.dtype), self._drv(t, B, Y.dtype, derivative=True)),
                           B, Y.dtype)

    def obs(self, t, Y, P):
        if self._obs is None:
            return np.zeros((Y.shape[0], 0), Y.dtype)
        B = Y.shape[0]
        return self._stack(self._obs(t, [Y[:, i] for i in range(self.n)], [P[:, j] for j in range(P.shape[1])],
                                     self._drv(t, B, Y.dtype)), B, Y.dtype)


class DriverTable:
    """Piecewise-polynomial drivers from a coefficient table
    ``[segment, driver, power]``, evaluated as the reference's device
    helpers do (array_interpolator.py:437-550): scaled time
    (t - start) / period with start = t0 - period for zero-padded clamped
    inputs, segment = floor (modulo the segment count when wrapping,
    clamped to the table otherwise), Horner in tau, zero outside the
    window when not wrapping; all in the working precision."""

    def __init__(self, coefficients, period, t0, wrap, padded, precision):
        p = np.dtype(precision).type
        self.p = p
        self.c = np.asarray(coefficients, dtype=p)
        self.nseg = self.c.shape[0]
        self.order = self.c.shape[2] - 1
        res = p(period)
        self.inv = p(p(1.0) / res)
        self.start = p(p(t0) - (res if padded else p(0.0)))
        self.wrap = bool(wrap)

    def evaluate(self, t, derivative=False):
        p = self.p
        scaled = (np.asarray(t, dtype=p) - self.start) * self.inv
        fl = np.floor(scaled)
        idx = fl.astype(np.int64)
        if self.wrap:
            seg = np.mod(idx, self.nseg)
            tau = (scaled - fl).astype(p)
            ok = np.ones(scaled.shape, bool)
        else:
            ok = (scaled >= 0) & (scaled <= self.nseg)
            seg = np.clip(idx, 0, self.nseg - 1)
            tau = (scaled - seg.astype(p)).astype(p)
        c = self.c[seg]
        acc = np.zeros((scaled.shape[0], self.c.shape[1]), p)
        if derivative:
            for k in range(self.order, 0, -1):
                acc = acc * tau[:, None] + p(k) * c[:, :, k]
            acc = acc * self.inv
        else:
            for k in range(self.order, -1, -1):
                acc = acc * tau[:, None] + c[:, :, k]
        return np.where(ok[:, None], acc, p(0))


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def pymax(a, b):
    return np.where(b > a, b, a)


def pymin(a, b):
    return np.where(b < a, b, a)


class Tol:
    """Tolerance vectors tiled to a solver width, in a given dtype."""

    def __init__(self, atol, rtol, dtype):
        self.atol = np.asarray(atol, dtype=dtype)
        self.rtol = np.asarray(rtol, dtype=dtype)


def scaled_norm2(v, ref, tol: Tol, ctype):
    """mean_i (|v_i| / max(atol + rtol |ref_i|, 1e-16))^2 (norms.py:180-196).
    ``v`` and ``ref`` have shape [B, K]; ``ref`` is tiled when narrower."""
    K = v.shape[1]
    n = ref.shape[1]
    reps = K // n
    reft = np.tile(ref, (1, reps)).astype(ctype)
    at = np.tile(tol.atol, reps).astype(ctype)
    rt = np.tile(tol.rtol, reps).astype(ctype)
    t = at + rt * np.abs(reft)
    t = pymax(t, ctype(1e-16))
    r = np.abs(v.astype(ctype)) / t
    return (r * r).sum(axis=1) * ctype(1.0 / K)


# ---------------------------------------------------------------------------
# Linear solvers (batched; ``A`` applies the operator to [B, K] vectors)
# ---------------------------------------------------------------------------
def mr_solve(A, P, norm2, rhs, x, floor, red, max_iters, sd, rt, ct):
    tol = ct(floor) + ct(red) * np.sqrt(norm2(rhs))
    tol2 = tol * tol
    rhs = rhs - A(x)
    acc = norm2(rhs)
    conv = acc <= tol2
    iters = np.zeros(rhs.shape[0], np.int64)
    for _ in range(max_iters):
        if conv.all():
            break
        act = ~conv
        iters += act
        z = P(rhs) if P is not None else rhs.copy()
        tmp = A(z)
        if sd:
            num = (rhs.astype(ct) * z).sum(1)
            den = (tmp.astype(ct) * z).sum(1)
        else:
            num = (tmp.astype(ct) * rhs).sum(1)
            den = (tmp.astype(ct) * tmp).sum(1)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = np.where(den != 0, num / np.where(den != 0, den, 1), 0).astype(rt)
        alpha = np.where(act, alpha, rt(0))
        x = x + alpha[:, None] * z
        rhs = rhs - alpha[:, None] * tmp
        acc = norm2(rhs)
        conv = conv | (acc <= tol2)
    status = np.where(conv, 0, 4)
    return x, status, iters


def bicgstab_solve(A, P, norm2, rhs, x, floor, red, max_iters, rt, ct):
    f32 = rt == np.float32
    tiny = rt(1e-30) if f32 else rt(1e-200)
    lim = rt(1e16) if f32 else rt(1e150)

    def cl(v):
        return np.clip(v, -lim, lim)

    tol = ct(floor) + ct(red) * np.sqrt(norm2(rhs))
    tol2 = tol * tol
    ax = cl(A(x))
    r = rhs - ax
    r0 = r.copy()
    p = cl(r)
    rho_prev = np.minimum(r * r, lim).sum(1)
    acc = norm2(r)
    conv = acc <= tol2
    broken = np.zeros_like(conv)
    fin = conv.copy()
    iters = np.zeros(r.shape[0], np.int64)
    with np.errstate(all="ignore"):
        for _ in range(max_iters):
            if fin.all():
                break
            iters += ~fin
            tmp = cl(P(p)) if P is not None else p.copy()
            v = cl(A(tmp))
            dot_r0v = cl(r0 * v).sum(1)
            a_over = np.abs(rho_prev) > np.abs(dot_r0v) * lim
            broken = broken | (~fin & a_over)
            fin = conv | broken
            alpha = np.where((dot_r0v != 0) & ~a_over, rho_prev / np.where(dot_r0v != 0, dot_r0v, 1), rt(0)).astype(rt)
            ae = np.where(fin, rt(0), alpha)
            x = x + ae[:, None] * tmp
            r = r - ae[:, None] * v
            acc = norm2(r)
            conv = conv | (acc <= tol2)
            fin = conv | broken
            sh = cl(P(r)) if P is not None else cl(r)
            tmp = cl(A(sh))
            dot_ts = cl(tmp * r).sum(1)
            dot_tt = np.minimum(tmp * tmp, lim).sum(1)
            o_over = np.abs(dot_ts) > dot_tt * lim
            omega = np.where((dot_tt != 0) & ~o_over, dot_ts / np.where(dot_tt != 0, dot_tt, 1), rt(0)).astype(rt)
            oe = np.where(fin, rt(0), omega)
            x = x + oe[:, None] * sh
            r = r - oe[:, None] * tmp
            acc = norm2(r)
            conv = conv | (acc <= tol2)
            rho_new = cl(r0 * r).sum(1)
            broken = broken | (~conv & ((np.abs(rho_new) < tiny) | (np.abs(omega) < tiny)))
            fin = conv | broken
            b_over = (np.abs(rho_new) > np.abs(rho_prev) * lim) | (np.abs(alpha) > np.abs(omega) * lim)
            broken = broken | (~fin & b_over)
            fin = conv | broken
            beta = np.where(~fin, (rho_new / rho_prev) * (alpha / omega), rt(0)).astype(rt)
            pn = r + beta[:, None] * (p - omega[:, None] * v)
            p = cl(np.where(fin[:, None], p, pn))
            rho_prev = np.where(fin, rho_prev, rho_new)
    status = np.where(conv, 0, np.where(broken, 128, 4))
    return x, status, iters


# ---------------------------------------------------------------------------
# the integrator
# ---------------------------------------------------------------------------
@dataclass
class Settings:
    precision: type = np.float32
    control_dtype: Optional[type] = None   # None: same as precision (reference mode)
    step_controller: Optional[str] = None
    dt: Optional[float] = None
    dt_min: Optional[float] = None
    dt_max: Optional[float] = None
    atol: float = 1e-6
    rtol: float = 1e-6
    kp: float = 0.7
    ki: float = -0.4
    kd: float = 0.0
    safety: float = 0.9
    min_gain: float = 0.3
    max_gain: float = 2.0
    deadband_min: float = 1.0
    deadband_max: float = 1.2
    newton_target_iters: int = 20
    linear_correction_type: str = "minimal_residual"
    krylov_max_iters: int = 100
    newton_max_iters: int = 100
    preconditioner_order: int = 2
    preconditioner_type: Optional[str] = "neumann"
    krylov_residual_reduction: Optional[float] = None
    save_every: Optional[float] = None
    summarise_every: Optional[float] = None
    sample_summaries_every: Optional[float] = None
    output_types: Sequence[str] = ("state",)
    dense_prediction: bool = True
    max_steps: int = 0
    # variable selection (output_config.py: saved_state_indices,
    # summarised_state_indices; summarise_variables by state name)
    saved_state_indices: Optional[Sequence[int]] = None
    summarised_state_indices: Optional[Sequence[int]] = None
    summarise_variables: Optional[Sequence[str]] = None


def integrate(system: OracleSystem, algorithm: str, inits: np.ndarray, params: np.ndarray,
              duration: float, settling_time: float = 0.0, t0: float = 0.0,
              durations: Optional[np.ndarray] = None, **kw) -> Dict[str, np.ndarray]:
    """Integrate every run (columns of ``inits``/``params``) and return the
    reference's outputs: ``state`` [save, var(+time), run], ``state_summaries``
    [summary, var*metric, run], ``iteration_counters`` [save, 4, run],
    ``status`` [run]."""
    S = Settings(**{k: v for k, v in kw.items() if k in Settings.__dataclass_fields__})
    extra = set(kw) - set(Settings.__dataclass_fields__)
    if extra:
        raise KeyError(f"unknown oracle settings {extra}")
    rt = np.dtype(S.precision).type
    ct = np.dtype(S.control_dtype).type if S.control_dtype is not None else rt
    mixed = ct != rt
    tab = TABLEAUS[algorithm]
    n = system.n
    if getattr(system, "mass", None) is not None and tab.kind == "erk":
        raise ValueError("a mass matrix needs an implicit algorithm")
    B = inits.shape[1]
    Y = np.ascontiguousarray(inits.T.astype(rt))
    P = np.ascontiguousarray(params.T.astype(rt)) if params.size else np.zeros((B, 0), rt)
    comp = np.zeros_like(Y)

    # controller settings (family defaults overridden by the caller)
    fam = dict(FAMILY_CONTROLLER[tab.kind]) if tab.has_err else {"step_controller": "fixed"}
    for key in ("step_controller", "kp", "ki", "kd", "safety", "min_gain", "max_gain", "deadband_min",
                "deadband_max"):
        v = kw.get(key)
        if v is not None:
            fam[key] = v
    ctl = fam.get("step_controller", "fixed")
    if not tab.has_err:
        ctl = "fixed"
    g = lambda k, d: fam.get(k, d)
    safety, min_gain, max_gain = g("safety", 0.9), g("min_gain", 0.3), g("max_gain", 2.0)
    db_min, db_max = g("deadband_min", 1.0), g("deadband_max", 1.2)
    kp, ki, kd = g("kp", 0.7), g("ki", -0.4), g("kd", 0.0)
    if ctl == "fixed":
        dt0 = S.dt if S.dt is not None else 1e-3
        dt_min = dt_max = dt0
    else:
        dt_min, dt_max, dt0 = S.dt_min, S.dt_max, S.dt
        if dt0 is not None:
            dt_min = dt_min if dt_min is not None else dt0 / 100
            dt_max = dt_max if dt_max is not None else dt0 * 100
        dt_min = 1e-6 if dt_min is None else dt_min
        dt_max = 1.0 if dt_max is None else dt_max
        dt0 = math.sqrt(dt_min * dt_max) if dt0 is None else dt0
        if dt0 < dt_min:
            dt_min = dt0 / 100
        if dt0 > dt_max:
            dt_max = dt0 * 100
    atol = np.full(n, S.atol, float) if np.ndim(S.atol) == 0 else np.asarray(S.atol, float)
    rtol = np.full(n, S.rtol, float) if np.ndim(S.rtol) == 0 else np.asarray(S.rtol, float)
    ctl_tol = Tol(atol, rtol, ct)
    kry_tol = Tol(atol, rtol, ct)
    new_tol = Tol(atol / 10.0, rtol / 10.0, ct)
    eps = float(np.finfo(rt).eps)
    floor = math.sqrt(eps)
    if S.krylov_residual_reduction is not None:
        red = S.krylov_residual_reduction
    elif tab.kind != "erk" and ctl != "fixed" and rtol.min() > 0:
        red = float(rtol.min()) * (0.01 if tab.kind == "rosenbrock" else 1.0)
    else:
        red = eps
    floor_c, red_c = ct(rt(floor)) if not mixed else ct(floor), ct(rt(red)) if not mixed else ct(red)

    def lin_solve(A, Pc, norm2, rhs, x):
        if S.linear_correction_type == "bicgstab":
            return bicgstab_solve(A, Pc, norm2, rhs, x, floor_c, red_c, S.krylov_max_iters, rt, ct)
        if S.linear_correction_type in ("gmres", "direct"):
            # GMRES has no reference counterpart; the oracle solves the small
            # dense system directly, which is the answer GMRES converges to.
            K = rhs.shape[1]
            eye = np.eye(K, dtype=rhs.dtype)
            M = np.stack([A(np.broadcast_to(eye[k], rhs.shape).copy()) for k in range(K)], axis=2)
            sol = np.linalg.solve(M.astype(np.float64), rhs.astype(np.float64)[:, :, None])[:, :, 0]
            return sol.astype(rhs.dtype), np.zeros(rhs.shape[0], np.int64), np.ones(rhs.shape[0], np.int64)
        return mr_solve(A, Pc, norm2, rhs, x, floor_c, red_c, S.krylov_max_iters,
                        S.linear_correction_type == "steepest_descent", rt, ct)

    # outputs and schedule
    ot = tuple(S.output_types)
    save_state = "state" in ot
    save_time = "time" in ot
    save_counters = "iteration_counters" in ot
    metrics = [m for m in ot if m.split("[")[0] in ("mean", "max", "min", "rms", "std", "extrema", "peaks",
                                                    "dxdt_max", "dxdt_min", "dxdt_extrema", "d2xdt2_max",
                                                    "d2xdt2_min", "d2xdt2_extrema")]
    time_domain = save_state or save_time or save_counters
    save_every = S.save_every if time_domain else None
    save_last = time_domain and save_every is None
    summarise = bool(metrics)
    sum_every, samp_every = S.summarise_every, S.sample_summaries_every
    if summarise:
        if sum_every is None:
            sum_every, samp_every = duration, duration / 100.0
        elif samp_every is None:
            samp_every = sum_every / 10.0
    else:
        sum_every = samp_every = None
    spp = int(round(float(rt(sum_every)) / float(rt(samp_every)))) if summarise else 1

    def count(dur, iv):
        tot = np.float64(rt(dur)) / np.float64(rt(iv))
        return int(np.floor(tot + min(4.0 * eps * tot, 0.49)))

    n_save = (count(duration, save_every) if save_every is not None else 0) + 1 + (1 if save_last else 0)
    start = np.float64(settling_time) + np.float64(t0)
    save_stop = start + (count(duration, save_every) + 0.5) * np.float64(rt(save_every)) if save_every else \
        start + np.float64(rt(duration))
    summ_stop = start + (count(duration, samp_every) + 0.5) * np.float64(rt(samp_every)) if summarise else \
        start + np.float64(rt(duration))
    n_summ = count(duration, samp_every) // spp if summarise else 0
    width = n + (1 if save_time else 0)
    out_state = np.zeros((max(n_save, 0), width, B), rt)
    out_cnt = np.zeros((max(n_save, 0), 4, B), np.int32)

    # summary buffers (one variable group per state)
    def mdef(m):
        name = m.split("[")[0]
        par = int(m.split("[")[1].split("]")[0]) if "[" in m else 0
        return name, par
    mlist = [mdef(m) for m in metrics]
    # metrics.py:345-467: requested pairs collapse into combined metrics
    for lo, hi, combo in (("max", "min", "extrema"), ("dxdt_max", "dxdt_min", "dxdt_extrema"),
                          ("d2xdt2_max", "d2xdt2_min", "d2xdt2_extrema")):
        if (lo, 0) in mlist and (hi, 0) in mlist:
            i = min(mlist.index((lo, 0)), mlist.index((hi, 0)))
            mlist = [x for x in mlist if x not in ((lo, 0), (hi, 0))]
            mlist.insert(i, (combo, 0))
    bsize = {"mean": 1, "max": 1, "min": 1, "rms": 1, "std": 3, "extrema": 2, "dxdt_max": 2, "dxdt_min": 2,
             "dxdt_extrema": 3, "d2xdt2_max": 3, "d2xdt2_min": 3, "d2xdt2_extrema": 4}
    osize = {"mean": 1, "max": 1, "min": 1, "rms": 1, "std": 1, "extrema": 2, "dxdt_max": 1, "dxdt_min": 1,
             "dxdt_extrema": 2, "d2xdt2_max": 1, "d2xdt2_min": 1, "d2xdt2_extrema": 2}
    buf_w = sum(3 + p if nm == "peaks" else bsize[nm] for nm, p in mlist)
    out_w = sum(p if nm == "peaks" else osize[nm] for nm, p in mlist)
    sbuf = np.zeros((B, n, max(buf_w, 1)), rt)
    out_summ = np.zeros((max(n_summ, 0), n * out_w, B), rt)

    def summ_update(mask, idx):
        vals = Y
        off = 0
        for nm, par in mlist:
            b = sbuf[:, :, off:]
            m2 = mask[:, None]
            if nm == "mean":
                b[:, :, 0] = np.where(m2, b[:, :, 0] + vals, b[:, :, 0])
            elif nm == "max":
                b[:, :, 0] = np.where(m2 & (vals > b[:, :, 0]), vals, b[:, :, 0])
            elif nm == "min":
                b[:, :, 0] = np.where(m2 & (vals < b[:, :, 0]), vals, b[:, :, 0])
            elif nm == "extrema":
                b[:, :, 0] = np.where(m2 & (vals > b[:, :, 0]), vals, b[:, :, 0])
                b[:, :, 1] = np.where(m2 & (vals < b[:, :, 1]), vals, b[:, :, 1])
            elif nm == "rms":
                s = np.where((idx == 0)[:, None], rt(0), b[:, :, 0])
                b[:, :, 0] = np.where(m2, s + vals * vals, b[:, :, 0])
            elif nm == "std":
                first = (idx == 0)[:, None] & m2
                b[:, :, 0] = np.where(first, vals, b[:, :, 0])
                b[:, :, 1] = np.where(first, rt(0), b[:, :, 1])
                b[:, :, 2] = np.where(first, rt(0), b[:, :, 2])
                sv = vals - b[:, :, 0]
                b[:, :, 1] = np.where(m2, b[:, :, 1] + sv, b[:, :, 1])
                b[:, :, 2] = np.where(m2, b[:, :, 2] + sv * sv, b[:, :, 2])
            elif nm.startswith("dxdt_"):
                # dxdt_{max,min,extrema}.py: unscaled first difference,
                # gated until one previous sample exists
                d = vals - b[:, :, 0]
                primed = m2 & (idx[:, None] >= 1)
                if nm in ("dxdt_max", "dxdt_extrema"):
                    b[:, :, 1] = np.where(primed & (d > b[:, :, 1]), d, b[:, :, 1])
                if nm == "dxdt_min":
                    b[:, :, 1] = np.where(primed & (d < b[:, :, 1]), d, b[:, :, 1])
                if nm == "dxdt_extrema":
                    b[:, :, 2] = np.where(primed & (d < b[:, :, 2]), d, b[:, :, 2])
                b[:, :, 0] = np.where(m2, vals, b[:, :, 0])
            elif nm.startswith("d2xdt2_"):
                # d2xdt2_{max,min,extrema}.py: unscaled second difference,
                # gated until two previous samples exist
                d = vals - rt(2.0) * b[:, :, 0] + b[:, :, 1]
                primed = m2 & (idx[:, None] >= 2)
                if nm in ("d2xdt2_max", "d2xdt2_extrema"):
                    b[:, :, 2] = np.where(primed & (d > b[:, :, 2]), d, b[:, :, 2])
                if nm == "d2xdt2_min":
                    b[:, :, 2] = np.where(primed & (d < b[:, :, 2]), d, b[:, :, 2])
                if nm == "d2xdt2_extrema":
                    b[:, :, 3] = np.where(primed & (d < b[:, :, 3]), d, b[:, :, 3])
                b[:, :, 1] = np.where(m2, b[:, :, 0], b[:, :, 1])
                b[:, :, 0] = np.where(m2, vals, b[:, :, 0])
            elif nm == "peaks":
                prev, pprev, pc = b[:, :, 0].copy(), b[:, :, 1].copy(), b[:, :, 2].astype(np.int64)
                hit = m2 & (idx[:, None] >= 2) & (pc < par) & (pprev != 0) & (prev > vals) & (pprev < prev)
                for q in range(par):
                    b[:, :, 3 + q] = np.where(hit & (pc == q), rt(1) * (idx[:, None] - 1), b[:, :, 3 + q])
                b[:, :, 2] = np.where(hit, (pc + 1).astype(rt), b[:, :, 2])
                b[:, :, 0] = np.where(m2, vals, b[:, :, 0])
                b[:, :, 1] = np.where(m2, prev, b[:, :, 1])
            off += 3 + par if nm == "peaks" else bsize[nm]

    def summ_save(mask, row):
        off = 0
        ooff = 0
        outs = np.zeros((B, n, max(out_w, 1)), rt)
        for nm, par in mlist:
            b = sbuf[:, :, off:]
            m2 = mask[:, None]
            if nm == "mean":
                outs[:, :, ooff] = (b[:, :, 0].astype(np.float64) / spp).astype(rt)
                b[:, :, 0] = np.where(m2, rt(0), b[:, :, 0])
            elif nm in ("max", "min"):
                outs[:, :, ooff] = b[:, :, 0]
                b[:, :, 0] = np.where(m2, rt(-1e30 if nm == "max" else 1e30), b[:, :, 0])
            elif nm == "extrema":
                outs[:, :, ooff] = b[:, :, 0]
                outs[:, :, ooff + 1] = b[:, :, 1]
                b[:, :, 0] = np.where(m2, rt(-1e30), b[:, :, 0])
                b[:, :, 1] = np.where(m2, rt(1e30), b[:, :, 1])
            elif nm == "rms":
                outs[:, :, ooff] = np.sqrt(b[:, :, 0].astype(np.float64) / spp).astype(rt)
                b[:, :, 0] = np.where(m2, rt(0), b[:, :, 0])
            elif nm == "std":
                ms = (b[:, :, 1].astype(np.float64) / spp).astype(rt)
                mss = (b[:, :, 2].astype(np.float64) / spp).astype(rt)
                var = mss - ms * ms
                with np.errstate(invalid="ignore"):
                    outs[:, :, ooff] = np.sqrt(var.astype(np.float64)).astype(rt)
                b[:, :, 0] = np.where(m2, b[:, :, 0] + ms, b[:, :, 0])
                b[:, :, 1] = np.where(m2, rt(0), b[:, :, 1])
                b[:, :, 2] = np.where(m2, rt(0), b[:, :, 2])
            elif nm.startswith("dxdt_") or nm.startswith("d2xdt2_"):
                first = nm.startswith("dxdt_")
                k0 = 1 if first else 2
                scale = rt(samp_every) if first else rt(samp_every) * rt(samp_every)
                hi_first = nm.endswith("_max") or nm.endswith("_extrema")
                outs[:, :, ooff] = b[:, :, k0] / scale
                b[:, :, k0] = np.where(m2, rt(-1e30) if hi_first else rt(1e30), b[:, :, k0])
                if nm.endswith("_extrema"):
                    outs[:, :, ooff + 1] = b[:, :, k0 + 1] / scale
                    b[:, :, k0 + 1] = np.where(m2, rt(1e30), b[:, :, k0 + 1])
            elif nm == "peaks":
                for q in range(par):
                    outs[:, :, ooff + q] = b[:, :, 3 + q]
                    b[:, :, 3 + q] = np.where(m2, rt(0), b[:, :, 3 + q])
                b[:, :, 2] = np.where(m2, rt(0), b[:, :, 2])
            off += 3 + par if nm == "peaks" else bsize[nm]
            ooff += par if nm == "peaks" else osize[nm]
        ok = mask & (row < n_summ)
        for r in np.where(ok)[0]:
            out_summ[row[r], :, r] = outs[r].reshape(-1)

    def save_rows(mask, idx, tp, counters):
        ok = mask & (idx < n_save)
        for r in np.where(ok)[0]:
            if save_state:
                out_state[idx[r], :n, r] = Y[r]
            if save_time:
                out_state[idx[r], width - 1, r] = rt(tp[r])
            if save_counters:
                out_cnt[idx[r], :, r] = counters[r]

    # loop state
    durs = np.full(B, float(duration)) if durations is None else np.asarray(durations, float)
    t = np.full(B, np.float64(t0))
    tp = t.astype(ct)
    t_end = (np.float64(settling_time) + np.float64(t0) + durs).astype(ct)
    sstop = np.full(B, save_stop) if durations is None else np.float64(settling_time) + np.float64(t0) + durs
    ustop = np.full(B, summ_stop) if durations is None else np.float64(settling_time) + np.float64(t0) + durs
    next_save = np.full(B, ct(settling_time + t0))
    next_upd = np.full(B, ct(settling_time + t0))
    save_idx = np.zeros(B, np.int64)
    summ_idx = np.zeros(B, np.int64)
    upd_idx = np.zeros(B, np.int64)
    counters = np.zeros((B, 4), np.int64)
    counters_total = np.zeros(B, np.int64)
    allm = np.ones(B, bool)
    if settling_time == 0.0:
        if save_every is not None:
            next_save = (next_save + ct(rt(save_every) if not mixed else save_every)).astype(ct)
        if summarise:
            next_upd = (ct(rt(samp_every) if not mixed else samp_every) + next_upd).astype(ct)
        save_rows(allm, save_idx, tp, counters)
        save_idx += 1
        if summarise:
            summ_save(allm, summ_idx)
    status = np.zeros(B, np.int64)
    it_status = np.zeros(B, np.int64)
    dt = np.full(B, ct(rt(dt0)) if not mixed else ct(dt0))
    dt_raw = dt.copy()
    stagn = np.zeros(B, np.int64)
    first = np.ones(B, bool)
    prev_acc = np.ones(B, bool)
    irrec = np.zeros(B, bool)
    done = np.zeros(B, bool)
    hist0 = np.zeros(B, ct)
    hist1 = np.zeros(B, ct)
    # step persistents
    s = tab.s
    if tab.kind == "erk":
        k_fsal = np.zeros((B, n), rt)
    ros_guess = np.zeros((B, n), rt)
    firk_u = np.zeros((B, s * n), rt)
    prev_dt_step = np.zeros(B, rt)
    theta_store = np.zeros(B, ct)
    dirk_z = np.zeros((B, n), rt)
    dirk_hist = np.zeros((B, s * n), rt)
    dense = S.dense_prediction and (tab.dense32 if rt == np.float32 else tab.dense64) > 0 and tab.kind in ("firk", "dirk")
    ratio_lim = rt(tab.dense32 if rt == np.float32 else tab.dense64)
    pc = _pred_coeffs(tab) if dense else None
    expo_scale = 2 * (tab.order + 1)
    save_reg = save_every is not None
    summ_reg = summarise
    SE = ct(rt(save_every)) if (save_reg and not mixed) else (ct(save_every) if save_reg else ct(0))
    UE = ct(rt(samp_every)) if (summ_reg and not mixed) else (ct(samp_every) if summ_reg else ct(0))
    a_r = tab.a.astype(rt)

    def predict(U, ratio, apply):
        first_pred = 1 if tab.a[0, 0] == 0.0 else 0
        Pw = pc.shape[0]
        T = np.zeros((B, s, s), rt)
        for r in range(first_pred, s):
            for cidx in range(s):
                acc = np.zeros(B, rt)
                for q in range(Pw - 1, -1, -1):
                    acc = acc * ratio + rt(pc[q, r, cidx])
                T[:, r, cidx] = acc * ratio
        out = U.copy()
        for k in range(n):
            prev = U[:, [c * n + k for c in range(s)]]
            for r in range(first_pred, s):
                val = (T[:, r, :] * prev).sum(1) if False else np.zeros(B, rt)
                accv = np.zeros(B, rt)
                for cidx in range(s):
                    accv = accv + T[:, r, cidx] * prev[:, cidx]
                out[:, r * n + k] = np.where(apply, accv, U[:, r * n + k])
        return out

    def newton(res_fn, jac_fn, op_builder, corr_norm2, u, theta_store, act):
        """Damped Newton (newton_krylov.py:340-517), batched."""
        prev_theta = np.where(theta_store > 0, theta_store, ct(1))
        ndz_prev = np.zeros(B, ct)
        conv = ~act.copy()
        failed = np.zeros(B, bool)
        last_lin = np.zeros(B, np.int64)
        iters = np.zeros(B, np.int64)
        kit = np.zeros(B, np.int64)
        stag_eps = ct(100.0) * ct(math.sqrt(eps))
        huge = ct(np.finfo(rt).max)
        for it in range(S.newton_max_iters):
            active = ~(conv | failed)
            if not active.any():
                break
            res = -res_fn(u)
            delta = np.zeros_like(u)
            A, Pc, nrm = op_builder(u)
            delta, lst, li = lin_solve(A, Pc, nrm, res, delta)
            kit += np.where(active, li, 0)
            last_lin = np.where(active, lst, last_lin)
            iters += active
            n2 = corr_norm2(delta, u)
            ndz = np.sqrt(n2).astype(ct)
            judged = active & (lst == 0)
            history = ndz_prev > 0
            with np.errstate(divide="ignore", invalid="ignore"):
                theta = np.where(history, pymax(ct(0.3) * prev_theta, ndz / np.where(history, ndz_prev, 1)), prev_theta)
            small_first = (iters == 1) & (ndz < ct(1e-5))
            eta_acc = (theta < 1) & (theta * ndz < ct(0.01) * (ct(1) - theta))
            nonfinite = ~(n2 <= huge)
            stagnant = judged & history & (np.abs(theta - 1) <= stag_eps)
            diverging = judged & ((history & (theta > 2)) | nonfinite)
            conv_st = stagnant & (ndz <= 1) & ~diverging
            failed_now = diverging | (stagnant & (ndz > 1))
            failed = failed | failed_now
            commit = judged & ~failed_now & ~conv_st
            u = np.where(commit[:, None], u + delta, u)
            conv = conv | conv_st | (commit & (eta_acc | small_first))
            ndz_prev = np.where(commit, ndz, ct(0))
            prev_theta = np.where(judged & history, theta, prev_theta)
        theta_out = np.where(conv, prev_theta, ct(1))
        fail_bits = np.where(failed, 256, 2)
        fail_bits = np.where(last_lin != 0, fail_bits | last_lin, fail_bits)
        st = np.where(conv, 0, fail_bits)
        st = np.where(act, st, 0)
        return u, st, iters, kit, np.where(act, theta_out, theta_store)

    def single_op(J, s_coef, ref):
        """A v = v - s J v and its Neumann preconditioner (order m)."""
        def A(v):
            return system.mv(v) - s_coef[:, None] * np.einsum("bij,bj->bi", J, v)

        def Pc(v):
            out = v.copy()
            for _ in range(S.preconditioner_order):
                out = v + s_coef[:, None] * np.einsum("bij,bj->bi", J, out)
            return out
        return A, (Pc if S.preconditioner_type == "neumann" else None), (lambda v: scaled_norm2(v, ref, kry_tol, ct))

    iteration = 0
    while True:
        iteration += 1
        active = ~done
        if not active.any():
            break
        end_of_step = (tp + dt_raw).astype(ct)
        if save_reg or summ_reg:
            finished = np.ones(B, bool)
            sfin = np.zeros(B, bool)
            ufin = np.zeros(B, bool)
            if save_reg:
                sfin = next_save.astype(np.float64) > sstop
                finished &= sfin
            if summ_reg:
                ufin = next_upd.astype(np.float64) > ustop
                finished &= ufin
        else:
            finished = end_of_step >= t_end
            sfin = ufin = np.zeros(B, bool)
        at_end = np.zeros(B, bool)
        if save_last:
            at_end = (tp < t_end) & finished
            finished = finished & ~at_end
        finished = finished | irrec
        if S.max_steps:
            # step budget (status bit 32), as the engine's ``max_steps``
            over = active & ~finished & (counters_total >= S.max_steps)
            status = np.where(over, status | 32, status)
            finished = finished | over
        done = done | (finished & active)
        act = ~done
        if not act.any():
            break
        do_save = ((end_of_step >= next_save) & ~sfin) if save_reg else np.zeros(B, bool)
        do_upd = ((end_of_step >= next_upd) & ~ufin) if summ_reg else np.zeros(B, bool)
        if save_last:
            do_save = do_save | at_end
        dt_eff = dt_raw.copy()
        trunc = np.zeros(B, bool)
        ev = do_save | do_upd
        if ev.any():
            ne = t_end.copy()
            if save_reg:
                ne = np.where(do_save, pymin(ne, next_save), ne).astype(ct)
            if summ_reg:
                ne = np.where(do_upd, pymin(ne, next_upd), ne).astype(ct)
            gap = (ne - tp).astype(ct)
            dte = np.where(gap > 0, gap, dt_raw)
            dt_eff = np.where(ev, dte, dt_raw).astype(ct)
            trunc = ev & (dt_eff != dt_raw)
        h = dt_eff.astype(rt)
        tt = tp.astype(rt)
        nit = np.zeros(B, np.int64)
        kitv = np.zeros(B, np.int64)
        step_status = np.zeros(B, np.int64)
        err = np.zeros((B, n), rt)
        # ------------------------------- steps -------------------------------
        if tab.kind == "erk":
            use_cached = (tab.a[-1] == tab.b).all() and tab.c[0] == 0 and tab.c[-1] == 1 and (~first & prev_acc)
            fy = system.f(tt, Y, P)
            k = np.where(use_cached[:, None], k_fsal, fy) if np.ndim(use_cached) else fy
            outacc = np.zeros((B, n), rt)
            erracc = np.zeros((B, n), rt)
            d = tab.d if tab.has_err else np.zeros(s)
            brow = tab.row_match(tab.b)
            bhrow = tab.row_match(tab.b_hat)
            outacc = outacc + rt(tab.b[0]) * k if brow is None else outacc
            erracc = erracc + rt(d[0]) * k if (tab.has_err and bhrow is None) else erracc
            acc = np.zeros((s - 1, B, n), rt)
            delta = np.zeros((B, n), rt)
            stage_states = {}
            for prev in range(s - 1):
                stage = prev + 1
                for succ in range(s - 1):
                    cf = tab.a[succ + 1, prev]
                    if cf != 0.0:
                        acc[succ] = acc[succ] + rt(cf) * k
                st_time = tt + h * rt(tab.c[stage])
                scaled = acc[prev] * h[:, None]
                if stage == brow:
                    delta = scaled
                acc[prev] = scaled + Y
                stage_states[stage] = acc[prev].copy()
                k = system.f(st_time, acc[prev], P)
                if brow is None:
                    outacc = outacc + rt(tab.b[stage]) * k
                if tab.has_err and bhrow is None:
                    erracc = erracc + rt(d[stage]) * k
            if brow is None:
                delta = outacc * h[:, None]
                ynew = delta + Y
            else:
                ynew = stage_states[brow]
            if tab.has_err:
                err = erracc * h[:, None] if bhrow is None else ynew - stage_states[bhrow]
            k_fsal = np.where(act[:, None], k, k_fsal)
        elif tab.kind == "rosenbrock":
            gamma = rt(tab.gamma)
            J = system.jac(tt, Y, P)
            tdv = system.dfdt(tt, Y, P) * h[:, None]
            with np.errstate(divide="ignore"):
                inv_dt = rt(1) / h
            hg = (gamma * h).astype(rt)
            A, Pc, nrm = single_op(J, hg, Y)
            fy = system.f(tt, Y, P)
            # The engine distributes h gamma where no reference result is
            # compared bit for bit (mixed precision, direct stage solves):
            # h gamma f + gamma sum_j C_sj K_j (+ gs h gamma (h f_t)), the
            # same sum in another order.
            folded = mixed or S.linear_correction_type == "direct"
            if folded:
                # (f_t is zero for autonomous systems: the term adds nothing)
                rhs = fy * hg[:, None] + (rt(tab.gamma_stages[0]) * tdv) * hg[:, None]
            else:
                rhs = ((fy + rt(tab.gamma_stages[0]) * tdv) * h[:, None]) * gamma
            Ks = []
            # the reference's Rosenbrock step never copies its Krylov count
            # into the step counters, so the reported counts stay zero
            x, st, li = lin_solve(A, Pc, nrm, rhs, ros_guess.copy())
            step_status |= st
            Ks.append(x)
            # generic_rosenbrock_w.py:526-745: the proposed state starts at y
            # and takes each weighted increment in turn, or is the stage state
            # whose row of a equals b; the error likewise
            brow = tab.row_match(tab.b)
            bhrow = tab.row_match(tab.b_hat)
            delta = x * rt(tab.b[0])
            ynew = Y + rt(tab.b[0]) * x if brow is None else Y.copy()
            err = x * rt(tab.d[0]) if bhrow is None else np.zeros_like(Y)
            for stage in range(1, s):
                st_time = tt + h * rt(tab.c[stage])
                Ys = Y.copy()
                for j in range(stage):
                    if tab.a[stage, j] != 0.0:
                        Ys = Ys + rt(tab.a[stage, j]) * Ks[j]
                if stage == brow:
                    ynew = Ys.copy()
                if stage == bhrow:
                    err = Ys.copy()
                fs = system.f(st_time, Ys, P)
                corr = np.zeros((B, n), rt)
                for j in range(stage):
                    if tab.C[stage, j] != 0.0:
                        corr = corr + rt(tab.C[stage, j]) * Ks[j]
                # with a mass matrix the C_ij K_j / h term is M (C_ij K_j) / h
                # (Hairer & Wanner, Solving ODEs II, VI.4); the reference
                # leaves M out of it (generic_rosenbrock_w.py:682-698), which
                # no non-identity M we tried survives
                if folded:
                    rhs = fs * hg[:, None] + gamma * system.mv(corr) + (rt(tab.gamma_stages[stage]) * tdv) * hg[:, None]
                else:
                    rv = fs + system.mv(corr) * inv_dt[:, None] + rt(tab.gamma_stages[stage]) * tdv
                    rhs = rv * h[:, None] * gamma
                x, st, li = lin_solve(A, Pc, nrm, rhs, Ks[stage - 1].copy())
                step_status |= st
                Ks.append(x)
                delta = delta + rt(tab.b[stage]) * x
                if brow is None:
                    ynew = ynew + rt(tab.b[stage]) * x
                if bhrow is None:
                    err = err + rt(tab.d[stage]) * x
            ros_guess = np.where(act[:, None], Ks[-1], ros_guess)
            if mixed and brow is None:
                # the engine's mixed mode forms the proposed state (which
                # only sizes the error tolerance) once from delta
                ynew = Y + delta
            if tab.has_err and bhrow is not None:
                err = ynew - err
        elif tab.kind == "firk":
            U = firk_u.copy()
            if dense:
                prev_dt = prev_dt_step.copy()
                prev_dt_step = np.where(act, h, prev_dt_step)
                safe = np.where(prev_dt > 0, prev_dt, h)
                ratio = (h / safe).astype(rt)
                apply = ~first & prev_acc & (ratio <= ratio_lim)
                U = predict(U, ratio, apply & act)

            def stage_states_of(u):
                out = []
                for i in range(s):
                    Ys = Y.copy()
                    for j in range(s):
                        if tab.a[i, j] != 0.0:
                            Ys = Ys + a_r[i, j] * u[:, j * n:(j + 1) * n]
                    out.append(Ys)
                return out

            def res_fn(u):
                out = np.zeros_like(u)
                for i, Ys in enumerate(stage_states_of(u)):
                    fi = system.f(tt + h * rt(tab.c[i]), Ys, P)
                    out[:, i * n:(i + 1) * n] = system.mv(u[:, i * n:(i + 1) * n]) - h[:, None] * fi
                return out

            def op_builder(u):
                Js = [system.jac(tt + h * rt(tab.c[i]), Ys, P) for i, Ys in enumerate(stage_states_of(u))]

                def cjv(v):
                    out = np.zeros_like(v)
                    for i in range(s):
                        w = np.zeros((B, n), rt)
                        for j in range(s):
                            if tab.a[i, j] != 0.0:
                                w = w + a_r[i, j] * v[:, j * n:(j + 1) * n]
                        out[:, i * n:(i + 1) * n] = np.einsum("bij,bj->bi", Js[i], w)
                    return out

                def A(v):
                    mv = np.concatenate([system.mv(v[:, i * n:(i + 1) * n]) for i in range(s)], axis=1)
                    return mv - h[:, None] * cjv(v)

                def Pc(v):
                    out = v.copy()
                    for _ in range(S.preconditioner_order):
                        out = v + h[:, None] * cjv(out)
                    return out
                return A, (Pc if S.preconditioner_type == "neumann" else None), \
                    (lambda v: scaled_norm2(v, Y, kry_tol, ct))

            def corr(delta_, u):
                tot = np.zeros(B, ct)
                for i, Ys in enumerate(stage_states_of(u)):
                    ref = pymax(np.abs(Ys), np.abs(Y)).astype(ct)
                    tol = pymax(new_tol.atol + new_tol.rtol * ref, ct(1e-16))
                    r = delta_[:, i * n:(i + 1) * n].astype(ct) / tol
                    tot = tot + (r * r).sum(1)
                return tot * ct(1.0 / (s * n))

            U, st, ni, ki_, theta_store = newton(res_fn, None, op_builder, corr, U, theta_store, act)
            firk_u = np.where(act[:, None], U, firk_u)
            step_status |= st
            nit += ni
            kitv += ki_
            brow = tab.row_match(tab.b)
            if brow is not None:
                delta = np.zeros((B, n), rt)
                yv = Y.copy()
                for j in range(s):
                    if tab.a[brow, j] != 0.0:
                        delta = delta + a_r[brow, j] * U[:, j * n:(j + 1) * n]
                        yv = yv + a_r[brow, j] * U[:, j * n:(j + 1) * n]
                ynew = yv
            else:
                delta = sum(rt(tab.b[j]) * U[:, j * n:(j + 1) * n] for j in range(s))
                ynew = Y + delta
            if tab.has_err:
                accv = np.zeros((B, n), rt)
                compv = np.zeros((B, n), rt)
                for j in range(s):
                    term = rt(tab.d[j]) * U[:, j * n:(j + 1) * n] - compv
                    tmp = accv + term
                    compv = (tmp - accv) - term
                    accv = tmp
                err = accv
        else:  # dirk
            if dense:
                prev_dt = prev_dt_step.copy()
                prev_dt_step = np.where(act, h, prev_dt_step)
                safe = np.where(prev_dt > 0, prev_dt, h)
                ratio = (h / safe).astype(rt)
                apply = ~first & prev_acc & (ratio <= ratio_lim)
                dirk_hist = predict(dirk_hist, ratio, apply & act)
            brow = tab.row_match(tab.b)
            bhrow = tab.row_match(tab.b_hat)
            d = tab.d if tab.has_err else np.zeros(s)
            base = Y.copy()
            outacc = np.zeros((B, n), rt)
            erracc = np.zeros((B, n), rt)
            accs = np.zeros((max(s - 1, 1), B, n), rt)
            z = dirk_z.copy()
            rhs_k = None
            delta = np.zeros((B, n), rt)
            ynew = np.zeros((B, n), rt)
            errrow = np.zeros((B, n), rt)
            for stage in range(s):
                st_time = tt + h * rt(tab.c[stage])
                if stage > 0:
                    prev = stage - 1
                    for succ in range(s - 1):
                        cf = tab.a[succ + 1, prev] if succ + 1 > prev else 0.0
                        if cf != 0.0:
                            accs[succ] = accs[succ] + rt(cf) * rhs_k
                    sdelta = accs[prev] * h[:, None]
                    base = sdelta + Y
                else:
                    sdelta = np.zeros((B, n), rt)
                aii = tab.a[stage, stage]
                if aii != 0.0:
                    if dense:
                        src = [0] * s
                        latest = {}
                        for st_i, nd in enumerate(tab.c):
                            src[st_i] = latest.get(nd, st_i)
                            latest[nd] = st_i
                        z = dirk_hist[:, src[stage] * n:(src[stage] + 1) * n].copy()
                    elif tab.euler_guess and stage > 0 and tab.a[stage - 1, stage - 1] == 0.0:
                        z = rhs_k * h[:, None]
                    a_c = rt(aii)
                    bb = base.copy()

                    def res_fn(zz, bb=bb, a_c=a_c, st_time=st_time):
                        return system.mv(zz) - h[:, None] * system.f(st_time, bb + a_c * zz, P)

                    def op_builder(zz, bb=bb, a_c=a_c, st_time=st_time):
                        J = system.jac(st_time, bb + a_c * zz, P)
                        return single_op(J, (a_c * h).astype(rt), bb)

                    def corr(dl, zz, bb=bb, a_c=a_c):
                        sv = bb + a_c * zz
                        ref = pymax(np.abs(sv), np.abs(Y)).astype(ct)
                        tol = pymax(new_tol.atol + new_tol.rtol * ref, ct(1e-16))
                        r = dl.astype(ct) / tol
                        return (r * r).sum(1) * ct(1.0 / n)

                    z, st, ni, ki_, theta_store = newton(res_fn, None, op_builder, corr, z, theta_store, act)
                    step_status |= st
                    # each stage's solve overwrites the step's counters
                    # (generic_dirk.py:640-652, newton_krylov.py:514-515)
                    nit = ni
                    kitv = ki_
                    if dense:
                        dirk_hist[:, stage * n:(stage + 1) * n] = np.where(
                            act[:, None], z, dirk_hist[:, stage * n:(stage + 1) * n])
                    base = base + a_c * z
                    sdelta = sdelta + a_c * z
                rhs_k = system.f(st_time, base, P)
                if dense and aii == 0.0:
                    # an explicit stage's increment h f joins the read-ahead
                    # history like a solved one (stage_predictors.py)
                    dirk_hist[:, stage * n:(stage + 1) * n] = np.where(
                        act[:, None], rhs_k * h[:, None], dirk_hist[:, stage * n:(stage + 1) * n])
                if brow is None:
                    outacc = outacc + rt(tab.b[stage]) * rhs_k
                elif brow == stage:
                    ynew = base.copy()
                    delta = sdelta
                if tab.has_err:
                    if bhrow is None:
                        erracc = erracc + rt(d[stage]) * rhs_k
                    elif bhrow == stage:
                        errrow = base.copy()
            dirk_z = np.where(act[:, None], z, dirk_z)
            if brow is None:
                delta = outacc * h[:, None]
                ynew = delta + Y
            if tab.has_err:
                err = erracc * h[:, None] if bhrow is None else ynew - errrow
        # ------------------------------ control ------------------------------
        first = np.where(act, False, first)
        it_status = np.where(act, it_status | step_status, it_status)
        failed = step_status != 0
        if ctl == "fixed":
            irrec = irrec | (act & failed)
        err = np.where(failed[:, None], rt(1e16), err)
        if ctl != "fixed":
            e = pymax(np.abs(err).astype(ct), ct(1e-16))
            tol = ctl_tol.atol + ctl_tol.rtol * pymax(np.abs(ynew).astype(ct), np.abs(Y).astype(ct))
            with np.errstate(all="ignore"):
                nrm2 = ((e / tol) ** 2).sum(1) * ct(1.0 / n)
            nrm2 = np.where(np.isnan(nrm2) | np.isinf(nrm2), ct(1e16), nrm2).astype(ct)
            accept = nrm2 <= 1
            with np.errstate(all="ignore"):
                if ctl == "i":
                    gain = ct(safety) * nrm2 ** (-ct(1.0 / expo_scale))
                elif ctl == "pi":
                    src = np.where(hist0 > 0, hist0, nrm2)
                    gain = ct(safety) * nrm2 ** (-ct(kp / expo_scale)) * src ** (-ct(ki / expo_scale))
                elif ctl == "pid":
                    eps_ = np.where(hist0 > 0, hist0, nrm2)
                    epps = np.where(hist1 > 0, hist1, eps_)
                    gain = ct(safety) * nrm2 ** (-ct(kp / expo_scale)) * eps_ ** (-ct(ki / expo_scale)) * \
                        epps ** (-ct(kd / expo_scale))
                else:
                    expo = ct(1.0 / expo_scale)
                    dtp = pymax(hist0, ct(1e-16))
                    erp = pymax(hist1, ct(1e-16))
                    numer = ct(1 + 2 * S.newton_target_iters) * ct(safety)
                    tmp = numer / (nit + 2 * S.newton_target_iters).astype(ct)
                    fac = np.where(ct(safety) < tmp, ct(safety), tmp)
                    gb = fac * nrm2 ** (-expo)
                    gg = ct(safety) * (dt / dtp) * (nrm2 * nrm2 / erp) ** (-expo)
                    gain = np.where(gg < gb, gg, gb)
                    gain = np.where(accept & (dtp > ct(1e-16)), gain, gb)
            gain = gain.astype(ct)
            gain = pymax(ct(min_gain), pymin(gain, ct(max_gain)))
            if not (db_min == 1.0 and db_max == 1.0):
                within = (gain >= ct(db_min)) & (gain <= ct(db_max))
                gain = np.where(within, ct(1), gain)
            gain = np.where(accept, gain, pymin(gain, ct(safety)))
            freeze = accept & trunc
            commit_h = accept & ~trunc & act
            dt_new_raw = (dt * gain).astype(ct)
            new_dt = np.where(freeze, dt, pymax(ct(dt_min), pymin(dt_new_raw, ct(dt_max))))
            if ctl == "pi":
                hist0 = np.where(commit_h, nrm2, hist0)
            elif ctl == "pid":
                hist1 = np.where(commit_h, hist0, hist1)
                hist0 = np.where(commit_h, nrm2, hist0)
            elif ctl == "gustafsson":
                hist0 = np.where(commit_h, dt, hist0)
                hist1 = np.where(commit_h, nrm2, hist1)
            dt = np.where(act, new_dt, dt).astype(ct)
            cst = np.where(freeze | (dt_new_raw > ct(dt_min)), 0, 8)
            accept = accept & ~failed
            it_status = np.where(act, it_status | cst, it_status)
            irrec = irrec | (act & (cst != 0))
        else:
            accept = ~failed
        dt_raw = np.where(act, dt, dt_raw)
        counters[:, 0] += np.where(act, nit, 0)
        counters[:, 1] += np.where(act, kitv, 0)
        counters[:, 2] += act
        counters_total += act
        counters[:, 3] += act & ~accept
        t_prop = t + dt_eff.astype(np.float64)
        stagn = np.where(act, np.where(t_prop == t, stagn + 1, 0), stagn)
        is_st = act & (stagn >= 2)
        it_status = np.where(is_st, it_status | 64, it_status)
        irrec = irrec | is_st
        status = np.where(act & irrec, status | it_status, status)
        acc_m = act & accept
        it_status = np.where(acc_m, 0, it_status)
        t = np.where(acc_m, t_prop, t)
        tp = t.astype(ct)
        if mixed:
            zc = delta + comp
            ys = Y + zc
            comp = np.where(acc_m[:, None], zc - (ys - Y), comp)
            Y = np.where(acc_m[:, None], ys, Y)
        else:
            Y = np.where(acc_m[:, None], ynew, Y)
        prev_acc = np.where(act, accept, prev_acc)
        do_save = do_save & acc_m
        do_upd = do_upd & acc_m
        if do_save.any():
            if save_reg:
                next_save = np.where(do_save, next_save + SE, next_save).astype(ct)
            save_rows(do_save, save_idx, tp, counters)
            save_idx = save_idx + do_save
            counters[do_save] = 0
        if do_upd.any():
            if summ_reg:
                next_upd = np.where(do_upd, next_upd + UE, next_upd).astype(ct)
            summ_update(do_upd, upd_idx)
            upd_idx = upd_idx + do_upd
            sv = do_upd & (upd_idx % spp == 0)
            if sv.any():
                summ_save(sv, summ_idx)
                summ_idx = summ_idx + sv
        if iteration > 10_000_000:
            raise RuntimeError("oracle loop did not terminate")
    if S.saved_state_indices is not None and save_state:
        keep = list(S.saved_state_indices) + ([width - 1] if save_time else [])
        out_state = out_state[:, keep, :]
    summ_sel = S.summarised_state_indices
    if S.summarise_variables is not None:
        summ_sel = [system.states.index(v) for v in S.summarise_variables]
    if summ_sel is not None and summarise:
        rows = out_summ.shape[0]
        out_summ = out_summ.reshape(rows, n, out_w, B)[:, list(summ_sel)].reshape(rows, len(summ_sel) * out_w, B)
    return dict(state=out_state, iteration_counters=out_cnt, state_summaries=out_summ,
                status=status.astype(np.int32), n_save=n_save, n_summ=n_summ)
