"""GPU checks of loop semantics that parity on final values can hide."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LORENZ = ["dx = sigma * (y - x)", "dy = x * (rho - z) - y", "dz = x * y - beta * z"]


def _lorenz(prec):
    from cubie_b200 import create_ODE_system
    return create_ODE_system(LORENZ, states={"x": 1.0, "y": 0.0, "z": 0.0}, parameters={"rho": 21.0},
                             constants={"sigma": 10.0, "beta": 8.0 / 3.0}, precision=prec)


@pytest.mark.parametrize("kernel", ["plain", "persistent"])
@pytest.mark.parametrize("prec", [np.float32, np.float64])
def test_saves_land_exactly_on_events(cuda_device, kernel, prec):
    """Steps are clamped onto save times (ode_loop.py:775-787)."""
    from cubie_b200 import Solver
    rng = np.random.default_rng(0)
    inits = rng.uniform(-10, 10, (3, 8))
    params = rng.uniform(20, 35, (1, 8))
    solver = Solver(_lorenz(prec), algorithm="dormand-prince-54", rtol=1e-7, atol=1e-9, save_every=0.1,
                    output_types=["state", "time"], kernel=kernel)
    res = solver.solve(inits, params, duration=0.5)
    t = res.time
    expected = np.arange(6) * 0.1
    np.testing.assert_allclose(t, np.repeat(expected[:, None], 8, axis=1), rtol=0, atol=4 * np.finfo(prec).eps)


def test_step_budget_sets_status_32(cuda_device):
    from cubie_b200 import Solver
    solver = Solver(_lorenz(np.float64), algorithm="dormand-prince-54", rtol=1e-8, atol=1e-10,
                    save_every=0.1, output_types=["state", "time"], max_steps=20)
    res = solver.solve(np.array([[1.0], [0.0], [0.0]]), np.array([[28.0]]), duration=1.0,
                       nan_error_trajectories=False)
    assert res.status_codes.tolist() == [32]
    assert res.totals["steps"] == 20
