"""FP64 forward-sensitivity reference for gradients of trajectory losses.

Test infrastructure (the checker of the engine's discrete adjoint, which has
no counterpart in the reference): integrates the state together with its
sensitivities to the initial state and the parameters,

    y' = f(t, y, p),  S_y' = J S_y,  S_p' = J S_p + df/dp,
    S_y(t0) = I,  S_p(t0) = 0,

with SciPy's DOP853 at a tight tolerance, one run at a time, and contracts
them with dL/dy at the save times:

    dL/dy0 = sum_r S_y(t_r)^T g_r,   dL/dp = sum_r S_p(t_r)^T g_r.
"""

from __future__ import annotations

from typing import Dict, Sequence

import numpy as np
import sympy as sp
from scipy.integrate import solve_ivp


class SensitivitySystem:
    """f, J = df/dy and df/dp from ``lhs = rhs`` equation strings."""

    def __init__(self, equations: Sequence[str], states: Sequence[str], parameters: Sequence[str],
                 constants: Dict[str, float] = None):
        constants = constants or {}
        t = sp.Symbol("t", real=True)
        table = {nm: sp.Symbol(nm, real=True) for nm in list(states) + list(parameters)}
        table.update({k: sp.Float(v, 17) for k, v in constants.items()})
        table["t"] = t
        derivs = {}
        for eq in equations:
            lhs, rhs = [x.strip() for x in eq.split("=", 1)]
            expr = sp.sympify(rhs, locals=table)
            if lhs.startswith("d") and lhs[1:] in states:
                derivs[lhs[1:]] = expr
            else:
                table[lhs] = expr
        ys = [table[s] for s in states]
        ps = [table[p] for p in parameters]
        f = sp.Matrix([derivs[s] for s in states])
        self.n, self.np = len(ys), len(ps)
        args = (t, ys, ps)
        self._f = sp.lambdify(args, list(f), "numpy")
        self._J = sp.lambdify(args, f.jacobian(sp.Matrix(ys)).tolist(), "numpy")
        self._P = sp.lambdify(args, f.jacobian(sp.Matrix(ps)).tolist(), "numpy") if ps else None

    def rhs(self, t, z, p):
        n, m = self.n, self.np
        y = z[:n]
        Sy = z[n:n + n * n].reshape(n, n)
        Sp = z[n + n * n:].reshape(n, m)
        f = np.asarray(self._f(t, list(y), list(p)), dtype=float)
        J = np.asarray(self._J(t, list(y), list(p)), dtype=float).reshape(n, n)
        dSy = J @ Sy
        dSp = J @ Sp + (np.asarray(self._P(t, list(y), list(p)), dtype=float).reshape(n, m) if m else 0.0)
        return np.concatenate([f, dSy.ravel(), np.asarray(dSp).ravel()])


def trajectory_gradients(system: SensitivitySystem, inits: np.ndarray, params: np.ndarray,
                         save_times: np.ndarray, grad_rows: np.ndarray, rtol: float = 1e-12,
                         atol: float = 1e-12):
    """States at ``save_times`` and dL/dy0, dL/dp for every run.

    ``inits`` [n, runs], ``params`` [m, runs], ``grad_rows`` [rows, n, runs]
    = dL/dy(t_r).  Returns (states [rows, n, runs], gy0 [n, runs], gp [m, runs]).
    """
    n, m = system.n, system.np
    runs = inits.shape[1]
    states = np.zeros((len(save_times), n, runs))
    gy0 = np.zeros((n, runs))
    gp = np.zeros((m, runs))
    for r in range(runs):
        z0 = np.concatenate([inits[:, r].astype(float), np.eye(n).ravel(), np.zeros(n * m)])
        p = params[:, r].astype(float)
        sol = solve_ivp(system.rhs, (float(save_times[0]), float(save_times[-1])), z0, method="DOP853",
                        t_eval=save_times, rtol=rtol, atol=atol, args=(p,))
        for k in range(len(save_times)):
            z = sol.y[:, k]
            Sy = z[n:n + n * n].reshape(n, n)
            Sp = z[n + n * n:].reshape(n, m)
            g = grad_rows[k, :, r]
            states[k, :, r] = z[:n]
            gy0[:, r] += Sy.T @ g
            if m:
                gp[:, r] += Sp.T @ g
    return states, gy0, gp
