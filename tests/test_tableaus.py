"""The algorithm registry against the reference's coefficient tables (no GPU).

``tests/golden/ref_tableaus.npz`` holds every tableau of the reference's
registries, written from its own modules by
``tests/golden/make_tableau_fixture.py``.  Each alias must exist here with
the same coefficients; the reference's single-purpose steps (explicit and
backward Euler, the predictor-corrector and Crank-Nicolson) must exist as
the tableaus that reproduce them; and every Runge-Kutta tableau must meet
its stated order on the Butcher conditions up to order four and on the
linear stability function up to its full order.
"""

from math import factorial
from pathlib import Path

import numpy as np
import pytest

from cubie_b200.tableaus import DIRK, ERK, FIRK, ROSENBROCK, TABLEAU_REGISTRY

FIXTURE = np.load(Path(__file__).resolve().parent / "golden" / "ref_tableaus.npz")
REF_ALIASES = sorted({k.split("/")[0] for k in FIXTURE.files})


def _ref(alias, field):
    key = f"{alias}/{field}"
    return FIXTURE[key] if key in FIXTURE.files else None


@pytest.mark.parametrize("alias", REF_ALIASES)
def test_registry_matches_reference_coefficients(alias):
    assert alias in TABLEAU_REGISTRY, f"missing algorithm alias {alias!r}"
    tab = TABLEAU_REGISTRY[alias]
    assert tab.kind == str(_ref(alias, "kind"))
    assert tab.order == int(_ref(alias, "order"))
    np.testing.assert_allclose(tab.a_matrix(), _ref(alias, "a"), rtol=0, atol=2e-15)
    np.testing.assert_allclose(tab.b, _ref(alias, "b"), rtol=0, atol=2e-15)
    np.testing.assert_allclose(tab.c, _ref(alias, "c"), rtol=0, atol=2e-15)
    if _ref(alias, "b_hat") is None:
        assert tab.b_hat is None
    else:
        np.testing.assert_allclose(tab.b_hat, _ref(alias, "b_hat"), rtol=0, atol=2e-15)
    assert tab.dense_ratio_float32 == float(_ref(alias, "dense32"))
    assert tab.dense_ratio_float64 == float(_ref(alias, "dense64"))
    if tab.kind == ROSENBROCK:
        s = tab.stage_count
        C = np.zeros((s, s))
        for i, row in enumerate(tab.C):
            C[i, :len(row)] = row
        np.testing.assert_allclose(C, _ref(alias, "C"), rtol=0, atol=2e-15)
        assert tab.gamma == pytest.approx(float(_ref(alias, "gamma")), abs=1e-16)
        np.testing.assert_allclose(tab.gamma_stages, _ref(alias, "gamma_stages"), rtol=0, atol=2e-16)


def test_single_purpose_steps_as_tableaus():
    """explicit_euler.py, backwards_euler.py, backwards_euler_predict_correct.py
    and crank_nicolson.py restated as tableaus."""
    eu = TABLEAU_REGISTRY["euler"]
    assert (eu.kind, eu.stage_count, eu.order, eu.has_error_estimate) == (ERK, 1, 1, False)
    assert eu.b == (1.0,)
    be = TABLEAU_REGISTRY["backwards_euler"]
    assert (be.kind, be.stage_count, be.b_row, be.has_error_estimate) == (DIRK, 1, 0, False)
    assert be.c == (1.0,) and be.dense_ratio_float32 == 0.0 == be.dense_ratio_float64
    pc = TABLEAU_REGISTRY["backwards_euler_pc"]
    assert pc.euler_guess and pc.first_same_as_last and pc.b_row == 1 and not pc.has_error_estimate
    cn = TABLEAU_REGISTRY["crank_nicolson"]
    assert cn.euler_guess and cn.order == 2 and cn.has_error_estimate
    assert (cn.b_row, cn.b_hat_row) == (1, 2)
    # only the step-start derivative is evaluated; the two solved stages
    # feed nothing that needs f at their states
    assert [cn.stage_derivative_needed(i) for i in range(3)] == [True, False, False]


def _rk_conditions(A, b, c, order):
    """Residuals of the Butcher order conditions for the rooted trees of
    order <= min(order, 4)."""
    e = np.ones_like(c)
    res = []
    checks = [
        (1, b @ e, 1.0),
        (2, b @ c, 1 / 2),
        (3, b @ c ** 2, 1 / 3),
        (3, b @ (A @ c), 1 / 6),
        (4, b @ c ** 3, 1 / 4),
        (4, b @ (c * (A @ c)), 1 / 8),
        (4, b @ (A @ c ** 2), 1 / 12),
        (4, b @ (A @ (A @ c)), 1 / 24),
    ]
    for p, val, want in checks:
        if p <= order:
            res.append(abs(val - want))
    return max(res)


def _stability_taylor(A, b, n):
    """Taylor coefficients of R(z) = 1 + z b^T (I - zA)^{-1} 1 up to z^n."""
    s = len(b)
    out = [1.0]
    v = np.ones(s)
    for _ in range(n):
        out.append(float(b @ v))
        v = A @ v
    return out


RK_ALIASES = sorted(k for k, t in TABLEAU_REGISTRY.items() if t.kind in (ERK, DIRK, FIRK))


@pytest.mark.parametrize("alias", RK_ALIASES)
def test_runge_kutta_order_conditions(alias):
    tab = TABLEAU_REGISTRY[alias]
    A = tab.a_matrix()
    b = np.asarray(tab.b)
    c = np.asarray(tab.c)
    np.testing.assert_allclose(A.sum(axis=1), c, atol=1e-12)
    assert _rk_conditions(A, b, c, tab.order) < 1e-12
    coeffs = _stability_taylor(A, b, tab.order)
    for k, v in enumerate(coeffs):
        assert v == pytest.approx(1.0 / factorial(k), abs=1e-12), (alias, k)
    if tab.has_error_estimate:
        # the embedded solution is consistent (at least first order)
        assert abs(np.sum(tab.b_hat) - 1.0) < 1e-12


def test_gauss_legendre_literals_follow_collocation():
    from cubie_b200.tableaus import _gauss_legendre
    for stages in (2, 4):
        built = _gauss_legendre(stages)
        tab = TABLEAU_REGISTRY[f"firk_gauss_legendre_{stages}"]
        np.testing.assert_allclose(tab.a_matrix(), built.a_matrix(), rtol=0, atol=2e-15)
        np.testing.assert_allclose(tab.b, built.b, rtol=0, atol=2e-15)
        np.testing.assert_allclose(tab.c, built.c, rtol=0, atol=2e-15)
