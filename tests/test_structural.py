"""DAE input through structural simplification (``create_ODE_system`` with
implicit equations, algebraic unknowns or second derivatives).

The expectations follow the reference's own tests of its structural
package (tests/odesystems/symbolic/structural/test_pipeline.py,
test_dae_parser.py, test_dae_solve.py): aliases and solvable algebraic
unknowns become observables, unsolvable ones stay as algebraic states with
their residuals under a singular mass matrix, second derivatives get a
companion state, and inconsistent systems raise.  The solves run the
generated kernel on the CPU (g++ host build) and, marked gpu, on the GPU.
"""

import numpy as np
import pytest
import sympy as sp

from cubie_b200 import Solver, create_ODE_system
from cubie_b200.structural import (ExtraEquationsSystemError, ExtraVariablesSystemError, InvalidSystemError,
                                   structural_simplify)

TORN = "dx = -z\n0 = z**5 + z - x"


def _deriv(sysm, name):
    return sysm.derivatives[name]


def _obs(sysm, name):
    return dict((a.name, e) for a, e in sysm.assignments)[name]


def _s(name):
    return sp.Symbol(name, real=True)


def test_torn_algebraic_unknown_keeps_a_residual_and_a_singular_mass():
    sysm = create_ODE_system(TORN, states={"x": 2.0, "z": 1.0}, precision=np.float64)
    assert sysm.state_names == ["x", "z"]
    assert np.array_equal(sysm.mass, np.diag([1.0, 0.0]))
    x, z = _s("x"), _s("z")
    assert sp.simplify(_deriv(sysm, "x") + z) == 0
    assert sp.simplify(_deriv(sysm, "z") - (z**5 + z - x)) == 0
    with pytest.raises(ValueError, match="implicit algorithm"):
        Solver(sysm, algorithm="euler")
    with pytest.raises(ValueError, match="cannot override"):
        create_ODE_system(TORN, states={"x": 2.0, "z": 1.0}, mass=np.diag([1.0, 0.0]))


def test_explicit_definitions_and_literal_implicit_lhs_become_observables():
    sysm = create_ODE_system(["dx = -k*x + y", "y = 2*x"], states={"x": 1.0}, observables=["y"],
                             parameters={"k": 0.5})
    assert sysm.state_names == ["x"] and sysm.observable_names == ["y"] and sysm.mass is None
    lit = create_ODE_system(["dx = -z", "0.0 = z + 2*x"], states={"x": 1.0, "z": 0.0})
    x = _s("x")
    assert lit.state_names == ["x"] and lit.mass is None
    assert "z" in lit.observable_names and sp.simplify(_obs(lit, "z") + 2 * x) == 0
    assert sp.simplify(_deriv(lit, "x") - 2 * x) == 0


def test_aliases_signs_and_priorities():
    x, y = _s("x"), _s("y")
    plain = create_ODE_system(["dx = -k*y", "0 = x - y"], states={"x": 1.0, "y": 1.0}, parameters={"k": 1.0})
    assert plain.state_names == ["x"] and _obs(plain, "y") == x
    neg = create_ODE_system(["dx = -k*y", "0 = x + y"], states={"x": 1.0, "y": 1.0}, parameters={"k": 1.0})
    assert _obs(neg, "y") == -x and sp.simplify(_deriv(neg, "x") - _s("k") * x) == 0
    pri = create_ODE_system(["dx = -3*x", "dy = -3*y", "0 = x - y"], states={"x": 1.0, "y": 1.0},
                            state_priority={"y": 5})
    assert pri.state_names == ["y"] and _obs(pri, "x") == y
    assert sp.simplify(_deriv(pri, "y") + 3 * y) == 0
    keep = create_ODE_system(["dx = -k*y", "y = x"], states={"x": 1.0, "y": 1.0}, parameters={"k": 1.0},
                             irreducible=["y"])
    assert "y" in keep.state_names and keep.mass is not None


def test_linear_block_solved_analytically_and_second_derivative_lowered():
    lin = create_ODE_system(["dx = -u", "0 = u + 2*v - x", "0 = 3*u - v - 1"],
                            states={"x": 1.0, "u": 0.0, "v": 0.0})
    x = _s("x")
    assert lin.state_names == ["x"] and sp.simplify(_obs(lin, "u") - (x + 2) / 7) == 0
    osc = create_ODE_system(["d(d(x, t), t) = -x"], states={"x": 1.0})
    assert osc.state_names == ["x", "x_t"] and osc.mass is None
    assert _deriv(osc, "x") == _s("x_t") and sp.simplify(_deriv(osc, "x_t") + x) == 0
    # a declared companion keeps its initial value
    osc2 = create_ODE_system(["d(d(x, t), t) = -x"], states={"x": 1.0, "x_t": 0.5})
    assert osc2.state_names == ["x", "x_t"] and osc2.initial_values["x_t"] == 0.5


def test_two_torn_residuals_pair_with_their_unknowns():
    sysm = create_ODE_system("dx = -z1\ndy = -z2\n0 = z1**5 + z1 - x\n0 = z2**3 + z2 - y",
                             states={"x": 1.0, "y": 1.0, "z1": 0.5, "z2": 0.5})
    assert sysm.state_names == ["x", "y", "z1", "z2"]
    assert [sysm.mass[i, i] for i in range(4)] == [1, 1, 0, 0]
    z1, z2 = _s("z1"), _s("z2")
    assert z1 in _deriv(sysm, "z1").free_symbols and z2 not in _deriv(sysm, "z1").free_symbols
    assert z2 in _deriv(sysm, "z2").free_symbols and z1 not in _deriv(sysm, "z2").free_symbols


def test_inconsistent_and_higher_index_systems_raise():
    with pytest.raises(ExtraVariablesSystemError):
        create_ODE_system(["dx = -z - w", "0 = z**3 - x"], states={"x": 1.0, "z": 0.0, "w": 0.0})
    with pytest.raises(ExtraEquationsSystemError):
        create_ODE_system(["dx = -x", "0 = x**2 - 1"], states={"x": 1.0}, simplify=True)
    # a constraint whose time derivative vanishes along the dynamics
    # cannot be reduced (x + y is conserved: the system is redundant)
    with pytest.raises(InvalidSystemError, match="vanishes identically"):
        create_ODE_system(["dx = z", "dy = -z", "0 = x + y - 1"], states={"x": 0.5, "y": 0.5, "z": 0.0})
    with pytest.raises(InvalidSystemError, match="derivatives of algebraic unknowns"):
        create_ODE_system(["dx = -z", "0 = dz + x"], states={"x": 1.0, "z": 0.0})
    with pytest.raises(ValueError, match="immutable"):
        create_ODE_system(["k = 2*x", "0 = z - k", "dx = -z"], states={"x": 1.0, "z": 0.0},
                          parameters={"k": 0.5})


def test_structural_simplify_plain_ode_passthrough():
    x, k = _s("x"), _s("k")
    res = structural_simplify([x], {x: -k * x}, [])
    assert res.states == [x] and res.mass_matrix is None and res.residuals == []
    # an explicit ODE given with simplify=True keeps its form
    sysm = create_ODE_system("dx = -k*x", states={"x": 1.0}, parameters={"k": 1.0}, simplify=True)
    assert sysm.state_names == ["x"] and sysm.mass is None


def _z_of_x(x):
    z = x / 2.0
    for _ in range(60):
        z = z - (z**5 + z - x) / (5.0 * z**4 + 1.0)
    return z


def _reduced_reference(x0, t_end, n):
    """RK4 on dx/dt = -z(x) with z from z**5 + z = x (the reference test's
    own check, test_dae_solve.py)."""
    dt, x = t_end / n, x0
    for _ in range(n):
        k1 = -_z_of_x(x)
        k2 = -_z_of_x(x + 0.5 * dt * k1)
        k3 = -_z_of_x(x + 0.5 * dt * k2)
        k4 = -_z_of_x(x + dt * k3)
        x = x + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6.0
    return x


def _torn_solver(algorithm, **kw):
    sysm = create_ODE_system(TORN, states={"x": 2.0, "z": 1.0}, precision=np.float64)
    base = dict(dt=1e-3, save_every=0.1, newton_atol=1e-10, newton_rtol=1e-10, krylov_residual_floor=1e-6,
                output_types=["state", "time"])
    base.update(kw)
    return Solver(sysm, algorithm=algorithm, **base)


@pytest.mark.parametrize("algorithm", ["backwards_euler", "radau"])
def test_torn_dae_solution_emulated(algorithm):
    """The torn DAE integrated by the generated kernel (host build):
    backward Euler at dt = 1e-3 within its O(dt) error of the reduced
    problem's solution, Radau IIA5 (adaptive, direct stage solves: the
    algebraic row leaves the coupled operator too ill-scaled for the
    default minimal-residual iteration) within 1e-6, and the constraint
    held at the saved points."""
    from host_emu.emu import run_emulated
    kw = {} if algorithm == "backwards_euler" else dict(rtol=1e-9, atol=1e-9, linear_correction_type="direct")
    solver = _torn_solver(algorithm, **kw)
    out = run_emulated(solver, np.array([[2.0], [1.0]]), np.zeros((0, 1)), 0.2)
    assert out["status"].tolist() == [0]
    x, z = out["state"][-1, 0, 0], out["state"][-1, 1, 0]
    x_ref = _reduced_reference(2.0, 0.2, 4000)
    bar = 2e-3 if algorithm == "backwards_euler" else 1e-6
    assert abs(x - x_ref) < bar and abs(z - _z_of_x(x_ref)) < bar
    assert abs(z**5 + z - x) < 1e-5


def test_robertson_implicit_form_matches_reference_mass_matrix_fixture():
    """Robertson kinetics written with its conservation law as an implicit
    equation: y3 is solved for (an observable) and the reduced ODE,
    integrated by the generated kernel (host build), agrees with the
    reference's own Radau run of the hand-formulated DAE (M = diag(1, 1, 0))
    within 10 tolerance units."""
    from pathlib import Path
    from host_emu.emu import run_emulated
    from cases import CASES, case_inputs
    case = CASES["rober_dae_radau_f64"]
    ref = np.load(Path(__file__).parent / "golden" / "ref_rober_dae_radau_f64.npz")
    sysm = create_ODE_system("dy1 = -k1*y1 + k3*y2*y3\ndy2 = k1*y1 - k3*y2*y3 - k2*y2**2\n0 = y1 + y2 + y3 - 1",
                             states={"y1": 1.0, "y2": 0.0, "y3": 0.0}, parameters=["k1", "k2", "k3"],
                             precision=np.float64)
    assert sysm.state_names == ["y1", "y2"] and "y3" in sysm.observable_names
    kw = dict(case["kwargs"], output_types=["state", "observables", "time"])
    solver = Solver(sysm, algorithm="radau", **kw)
    inits, params = case_inputs(case)
    out = run_emulated(solver, inits[:2], params, case["duration"])
    assert out["status"].tolist() == [0] * inits.shape[1]
    mine = np.concatenate([out["state"][:, :2, :], out["obs"][:, :1, :]], axis=1)
    theirs = ref["state"][:, :3, :]
    units = np.abs(mine - theirs) / (kw["atol"] + kw["rtol"] * np.abs(theirs))
    assert float(np.max(units)) < 10.0


@pytest.mark.gpu
@pytest.mark.parametrize("algorithm", ["backwards_euler", "radau"])
def test_torn_dae_solution_gpu(cuda_device, algorithm):
    kw = {} if algorithm == "backwards_euler" else dict(rtol=1e-9, atol=1e-9, linear_correction_type="direct")
    r = _torn_solver(algorithm, **kw).solve(np.array([[2.0], [1.0]]), np.zeros((0, 1)), duration=0.2,
                                            nan_error_trajectories=False)
    assert r.status_codes.tolist() == [0]
    x, z = float(r.state[-1, 0, 0]), float(r.state[-1, 1, 0])
    x_ref = _reduced_reference(2.0, 0.2, 4000)
    bar = 2e-3 if algorithm == "backwards_euler" else 1e-6
    assert abs(x - x_ref) < bar and abs(z - _z_of_x(x_ref)) < bar
    assert abs(z**5 + z - x) < 1e-5


def test_structural_helpers():
    """The matching, component ordering and alias detection on small
    hand-made cases."""
    from cubie_b200.structural import _alias, _components, _match
    x, y, z = _s("x"), _s("y"), _s("z")
    assert _alias(x - y, {x, y}) in ((x, y, 1), (y, x, 1))
    assert _alias(x + y, {x, y})[2] == -1
    assert _alias(2 * x - y, {x, y}) is None and _alias(x - y + 1, {x, y}) is None
    # equations {x, y}, {y}, {y, z}: the only complete matching is x, y, z
    assert _match([{x, y}, {y}, {y, z}], [x, y, z]) == [0, 1, 2]
    assert _match([{x}, {x}], [x, y]) is None
    # 0 -> 1 -> 2 -> 1: components {1, 2} before {0}
    assert _components(3, [[1], [2], [1]]) == [[1, 2], [0]]


PENDULUM = "dx = vx\ndy = vy\ndvx = T*x\ndvy = T*y - g\n0 = x**2 + y**2 - L**2"
PENDULUM_STATES = {"x": 1.0, "y": 0.0, "vx": 0.0, "vy": 0.0, "T": 0.0}


def test_pendulum_index_reduction_and_state_selection():
    """The Cartesian pendulum (index 3): the constraint is differentiated
    twice along the dynamics, its two lower derivatives stay as invariants
    and demote one state each; with priorities on y and vy the solver
    keeps y and vy, x stays as an algebraic state under x^2 + y^2 = L^2,
    and vx and the tension T are solved for (observables)."""
    sysm = create_ODE_system(PENDULUM, states=PENDULUM_STATES, constants={"g": 9.81, "L": 1.0},
                             state_priority={"y": 10, "vy": 10}, precision=np.float64)
    assert sysm.state_names == ["y", "vy", "x"]
    assert [sysm.mass[i, i] for i in range(3)] == [1, 1, 0]
    assert {"vx", "T"} <= set(sysm.observable_names)
    x, y, vy = _s("x"), _s("y"), _s("vy")
    assert sp.simplify(_deriv(sysm, "x") - (x**2 + y**2 - _s("L") ** 2)) == 0
    assert sp.simplify(_obs(sysm, "vx") + vy * y / x) == 0
    with pytest.raises(ValueError, match="implicit algorithm"):
        Solver(sysm, algorithm="dormand-prince-54")
    # without priorities the later-declared states are demoted
    plain = create_ODE_system(PENDULUM, states=PENDULUM_STATES, constants={"g": 9.81, "L": 1.0})
    assert plain.state_names == ["x", "vx", "y"] and {"vy", "T"} <= set(plain.observable_names)


def _pendulum_reference(ts):
    """Minimal coordinates: x = cos(phi), y = -sin(phi), phi'' = g cos(phi)."""
    from scipy.integrate import solve_ivp as scipy_ivp
    ref = scipy_ivp(lambda t, z: [z[1], 9.81 * np.cos(z[0])], (0.0, float(ts[-1])), [0.0, 0.0], rtol=1e-12,
                    atol=1e-12, dense_output=True)
    phi, dphi = ref.sol(ts)
    return -np.sin(phi), -np.cos(phi) * dphi, np.cos(phi)


def _pendulum_solver():
    sysm = create_ODE_system(PENDULUM, states=PENDULUM_STATES, constants={"g": 9.81, "L": 1.0},
                             state_priority={"y": 10, "vy": 10}, precision=np.float64)
    return sysm, Solver(sysm, algorithm="radau", rtol=1e-10, atol=1e-10, linear_correction_type="direct",
                        output_types=["state", "time"], save_every=0.05, dt_min=1e-14)


def test_pendulum_solution_emulated():
    """The index-reduced pendulum through the generated kernel (host build),
    Radau IIA5, over t in [0, 0.3] (x stays away from 0, where the static
    selection would turn singular): positions and velocity within 1e-8 of
    the minimal-coordinates solution, the constraint held to rounding."""
    from host_emu.emu import run_emulated
    sysm, solver = _pendulum_solver()
    x0 = np.array([[sysm.initial_values[n]] for n in sysm.state_names])
    out = run_emulated(solver, x0, np.zeros((0, 1)), 0.3)
    assert out["status"].tolist() == [0]
    st = out["state"][:, :, 0]
    y_ref, vy_ref, x_ref = _pendulum_reference(st[:, -1])
    assert np.max(np.abs(st[:, 0] - y_ref)) < 1e-8 and np.max(np.abs(st[:, 1] - vy_ref)) < 1e-8
    assert np.max(np.abs(st[:, 2] - x_ref)) < 1e-8
    assert np.max(np.abs(st[:, 2] ** 2 + st[:, 0] ** 2 - 1.0)) < 1e-12


@pytest.mark.gpu
def test_pendulum_solution_gpu(cuda_device):
    sysm, solver = _pendulum_solver()
    x0 = np.array([[sysm.initial_values[n]] for n in sysm.state_names])
    r = solver.solve(x0, np.zeros((0, 1)), duration=0.3, nan_error_trajectories=False)
    assert r.status_codes.tolist() == [0]
    st = r.state[:, :, 0]
    y_ref, vy_ref, x_ref = _pendulum_reference(st[:, -1])
    assert np.max(np.abs(st[:, 0] - y_ref)) < 1e-8 and np.max(np.abs(st[:, 1] - vy_ref)) < 1e-8
    assert np.max(np.abs(st[:, 2] ** 2 + st[:, 0] ** 2 - 1.0)) < 1e-12
