"""Algorithmic floating-point work of an integration, for roofline statements.

The count combines the operation counts of the generated system functions
(:mod:`cubie_b200.codegen` counts adds, multiplies, divisions and special
calls on the common-subexpression DAG) with the iteration totals a launch
reports (attempted steps, Newton iterations, Krylov iterations).  Vector
work is counted as the arithmetic the algorithm needs, one flop per add,
multiply or divide on each element:

* weighted norm of a vector of width K: 7 K (tolerance a + r|y|, max,
  divide, square, accumulate);
* operator application ``v - s J v``: ``jmv`` + 2 K; the coupled S-stage
  operator adds the stage coupling ``sum_j a_ij v_j`` (2 S K);
* one GMRES (Arnoldi) iteration at basis index j: scaling in and out
  (12 K), one operator application, modified Gram-Schmidt (4 K (j + 1)),
  normalisation (3 K), Givens rotations (6 j + 6); per solve, the initial
  residual and norms (2 weighted norms, one application) and the solution
  update (2 K per basis vector + 7 K);
* MR/SD iteration: preconditioner (order m applications), one application,
  two dot products (4 K), two axpys (4 K), one weighted norm;
* direct solve (dense LU with partial pivoting; for K = 2 the closed-form
  inverse): forming the operator from K applications, factoring (sum over
  pivots of one reciprocal and 2 (K-k-1)^2 + (K-k-1) for the eliminations;
  8 for the 2 x 2 inverse), and 2 K^2 per solve (6 for K = 2); a
  Rosenbrock step factors once and solves every stage;
* the step-size controller: 9 N plus two powers.

The result is the work the method performs, not the instruction count the
GPU issues (integer indexing, predication and control flow are excluded).
"""

from __future__ import annotations

from typing import Dict

from .codegen import FlopCount
from .tableaus import DIRK, ERK, FIRK, ROSENBROCK


def _f(flops: Dict[str, FlopCount], name: str) -> int:
    return flops[name].flops if name in flops else 0


def direct_factor_flops(K: int, op_flops: int) -> float:
    if K == 2:
        # closed-form inverse: determinant (3), reciprocal (1), four scaled
        # entries (4)
        return K * op_flops + 8
    elim = sum(1 + 2 * (K - k - 1) ** 2 + (K - k - 1) for k in range(K))
    return K * op_flops + elim


def linear_iteration_flops(lin: str, K: int, op_flops: int, precond_order: int, preconditioned: bool,
                           restart: int) -> float:
    if lin == "direct":
        # K = 2: two multiplies and two multiply-adds
        return 6 if K == 2 else 2 * K * K
    if lin == "gmres":
        m = min(restart, K)
        j_avg = (m - 1) / 2.0
        pre = precond_order * (op_flops + K) if preconditioned else 0
        return 12 * K + op_flops + pre + 4 * K * (j_avg + 1) + 3 * K + 6 * j_avg + 6
    pre = precond_order * (op_flops + K) if preconditioned else 0
    if lin == "bicgstab":
        return 2 * (op_flops + pre) + 20 * K + 2 * 7 * K
    return op_flops + pre + 8 * K + 7 * K


def linear_solve_overhead(lin: str, K: int, op_flops: int, restart: int) -> float:
    if lin == "direct":
        return direct_factor_flops(K, op_flops)
    if lin == "gmres":
        m = min(restart, K)
        return 2 * 7 * K + op_flops + K + 2 * K * m + 7 * K + m * m
    return 7 * K + op_flops + K + 7 * K


def estimate_flops(spec, gen, totals: Dict[str, int]) -> float:
    """Algorithmic FLOPs of a launch from its iteration totals."""
    tab = spec.tableau
    n = gen.n
    S = tab.stage_count
    fl = gen.flops
    rhs, jac, jmv, dfdt = _f(fl, "dxdt"), _f(fl, "jac"), _f(fl, "jmv"), _f(fl, "dfdt")
    steps = totals["steps"]
    newton = totals["newton"]
    krylov = totals["krylov"]
    lin = spec.linear_correction_type
    ctrl = 9 * n + 2 if spec.controller != "fixed" else 0
    comp = 4 * n if spec.mixed_precision else 0
    if tab.kind == ERK:
        per_step = S * rhs + 2 * n * sum(1 for i in range(S) for j in range(S) if tab.a_matrix()[i, j] != 0)
        per_step += 4 * n * S + 2 * n
        return steps * (per_step + ctrl + comp)
    if tab.kind == ROSENBROCK:
        K = n
        op = jmv + 2 * K
        per_step = jac + dfdt + n + S * rhs + S * 12 * n + 4 * n * S + n
        solves = steps * S
        it = linear_iteration_flops(lin, K, op, spec.preconditioner_order, spec.preconditioned, spec.gmres_restart)
        if lin == "direct":
            return steps * (per_step + ctrl + comp + direct_factor_flops(K, op)) + krylov * it
        return steps * (per_step + ctrl + comp) + solves * linear_solve_overhead(lin, K, op, spec.gmres_restart) \
            + krylov * it
    if tab.kind == FIRK:
        K = S * n
        op = S * (2 * S * n + jmv) + 2 * K
        stage_states = S * 2 * S * n
        per_newton = (stage_states + S * (rhs + 2 * n)) + (stage_states + S * jac) + (stage_states + 10 * K) + K
        per_step = 4 * S * n + 2 * n + (S * S * 4 * n if spec.dense_prediction is not False else 0)
        it = linear_iteration_flops(lin, K, op, spec.preconditioner_order, spec.preconditioned, spec.gmres_restart)
        return steps * (per_step + ctrl + comp) + newton * (per_newton + linear_solve_overhead(
            lin, K, op, spec.gmres_restart)) + krylov * it
    # DIRK
    K = n
    op = jmv + 2 * K
    per_newton = (2 * n + rhs + n) + (2 * n + jac) + 10 * n + n
    per_step = S * (rhs + 4 * n) + 2 * n * S * S
    it = linear_iteration_flops(lin, K, op, spec.preconditioner_order, spec.preconditioned, spec.gmres_restart)
    return steps * (per_step + ctrl + comp) + newton * (per_newton + linear_solve_overhead(
        lin, K, op, spec.gmres_restart)) + krylov * it
