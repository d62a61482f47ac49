"""The adjoint kernels' arithmetic, checked on the CPU: the generated
translation unit with the adjoint kernels is compiled by g++ through the
host-emulation harness and compared with the FP64 forward-sensitivity
reference (oracle/sensitivity.py)."""

import numpy as np
import pytest

FHN = ["dV = V - V**3 / 3 - w + I", "dw = (V + a - b * w) / tau"]
VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]


def _run(eqs, states, params, x0, p, T, algorithm, **kw):
    from host_emu.emu import run_emulated_adjoint
    from cubie_b200 import Solver, create_ODE_system
    from oracle.sensitivity import SensitivitySystem, trajectory_gradients
    rng = np.random.default_rng(9)
    target = rng.uniform(-1.0, 1.0, (int(T) + 1, x0.shape[1]))

    def grad_fn(state):
        g = np.zeros(state.shape)
        g[:, 0, :] = 2.0 * (state[:, 0, :].astype(np.float64) - target) / target.size
        return g

    sysm = create_ODE_system(eqs, states={s: 0.0 for s in states}, parameters={q: 1.0 for q in params},
                             precision=np.float64)
    solver = Solver(sysm, algorithm=algorithm, output_types=["state"], save_every=1.0, adjoint=True, **kw)
    state, status, gi, gp = run_emulated_adjoint(solver, x0, p, T, grad_fn, max_ckpts=512)
    ssys = SensitivitySystem(eqs, states, params)
    _, gy0, gpr = trajectory_gradients(ssys, x0, p, np.arange(int(T) + 1, dtype=float), grad_fn(state))
    assert np.all(status == 0)
    return (np.max(np.abs(gi - gy0)) / np.max(np.abs(gy0)), np.max(np.abs(gp - gpr)) / np.max(np.abs(gpr)))


def test_erk_adjoint_emulated():
    rng = np.random.default_rng(1)
    x0 = np.stack([rng.uniform(-1, 1, 3), rng.uniform(-0.5, 0.5, 3)])
    p = np.stack([rng.uniform(0.5, 0.9, 3), rng.uniform(0.6, 1.0, 3), rng.uniform(8, 15, 3), rng.uniform(0.3, 0.6, 3)])
    ri, rp = _run(FHN, ["V", "w"], ["a", "b", "tau", "I"], x0, p, 8.0, "dormand-prince-54", rtol=1e-10, atol=1e-10)
    assert ri < 1e-7 and rp < 1e-7


def test_rosenbrock_adjoint_emulated():
    rng = np.random.default_rng(2)
    x0 = rng.uniform(-2, 2, (2, 3))
    p = (10.0 ** rng.uniform(0, 1, 3))[None, :]
    ri, rp = _run(VDP, ["x", "y"], ["mu"], x0, p, 5.0, "ros3p", rtol=1e-9, atol=1e-9,
                  linear_correction_type="gmres", preconditioner_type=None)
    assert ri < 1e-5 and rp < 1e-5


def test_erk_tape_replay_is_exact_with_time_dependence_and_rejections():
    """The explicit adjoint replays segments from the step-size tape.  A
    forced, time-dependent system at a loose tolerance (rejected attempts,
    so first-stage re-evaluations) must give gradients that do not depend on
    the checkpoint spacing at all (every spacing reconstructs the forward's
    steps exactly), and that agree with the FP64 forward sensitivities to
    the forward's own accuracy."""
    from host_emu.emu import run_emulated_adjoint
    from cubie_b200 import Solver, create_ODE_system
    from oracle.sensitivity import SensitivitySystem, trajectory_gradients
    eqs = ["dV = V - V**3 / 3 - w + I * (1 + 0.3 * sin(0.5 * t))", "dw = (V + a - b * w) / tau"]
    states, params = ["V", "w"], ["a", "b", "tau", "I"]
    rng = np.random.default_rng(5)
    x0 = np.stack([rng.uniform(-1, 1, 3), rng.uniform(-0.5, 0.5, 3)])
    p = np.stack([rng.uniform(0.5, 0.9, 3), rng.uniform(0.6, 1.0, 3), rng.uniform(8, 15, 3), rng.uniform(0.3, 0.6, 3)])
    T = 30.0
    target = rng.uniform(-1.0, 1.0, (int(T) + 1, 3))

    def grad_fn(state):
        g = np.zeros(state.shape)
        g[:, 0, :] = 2.0 * (state[:, 0, :].astype(np.float64) - target) / target.size
        return g

    sysm = create_ODE_system(eqs, states={s: 0.0 for s in states}, parameters={q: 1.0 for q in params},
                             precision=np.float64)
    solver = Solver(sysm, algorithm="dormand-prince-54", output_types=["state"], save_every=1.0, adjoint=True,
                    rtol=1e-5, atol=1e-5, dt=1.0)
    results = [run_emulated_adjoint(solver, x0, p, T, grad_fn, ckpt_every=ce, max_ckpts=512)
               for ce in (1, 5, 64)]
    for state, status, gi, gp in results:
        assert np.all(status == 0)
        np.testing.assert_array_equal(gi, results[0][2])
        np.testing.assert_array_equal(gp, results[0][3])
    ssys = SensitivitySystem(eqs, states, params)
    _, gy0, gpr = trajectory_gradients(ssys, x0, p, np.arange(int(T) + 1, dtype=float), grad_fn(results[0][0]))
    gi, gp = results[0][2], results[0][3]
    assert np.max(np.abs(gi - gy0)) / np.max(np.abs(gy0)) < 2e-3
    assert np.max(np.abs(gp - gpr)) / np.max(np.abs(gpr)) < 2e-3


def test_erk_adjoint_with_array_driver_matches_finite_differences():
    """Explicit adjoint of a system forced through the array interpolator (the
    tape keeps control-precision step sizes and the record keeps stage
    times): parameter gradients against central differences of the FP64
    forward loss, and spacing-independent to the bit."""
    from host_emu.emu import run_emulated, run_emulated_adjoint
    from cubie_b200 import Solver, create_ODE_system
    eqs = ["dV = V - V**3 / 3 - w + drive", "dw = (V + a - b * w) / tau"]
    rng = np.random.default_rng(8)
    n = 2
    x0 = np.stack([rng.uniform(-1, 1, n), rng.uniform(-0.5, 0.5, n)])
    p = np.stack([rng.uniform(0.5, 0.9, n), rng.uniform(0.6, 1.0, n), rng.uniform(8, 15, n)])
    T = 12.0
    t_s = np.arange(200) * 0.1
    drv = {"driver_sample_period": 0.1, "t0": 0.0, "order": 3, "wrap": False,
           "drive": 0.5 + 0.3 * np.sin(0.7 * t_s)}
    target = rng.uniform(-1.0, 1.0, (int(T) + 1, n))

    def loss_grad(state):
        g = np.zeros(state.shape)
        g[:, 0, :] = 2.0 * (state[:, 0, :] - target) / target.size
        return g

    sysm = create_ODE_system(eqs, states={"V": 0.0, "w": 0.0}, parameters={"a": 0.7, "b": 0.8, "tau": 12.5},
                             drivers=["drive"], precision=np.float64)
    solver = Solver(sysm, algorithm="dormand-prince-54", output_types=["state"], save_every=1.0, adjoint=True,
                    rtol=1e-10, atol=1e-10)
    runs = [run_emulated_adjoint(solver, x0, p, T, loss_grad, ckpt_every=ce, max_ckpts=4096, drivers=drv)
            for ce in (1, 64)]
    for state, status, gi, gp in runs:
        assert np.all(status == 0)
        np.testing.assert_array_equal(gp, runs[0][3])
        np.testing.assert_array_equal(gi, runs[0][2])
    gp = runs[0][3]
    plain = Solver(sysm, algorithm="dormand-prince-54", output_types=["state"], save_every=1.0, rtol=1e-10,
                   atol=1e-10)

    def loss(pp):
        st = run_emulated(plain, x0, pp, T, drivers=drv)["state"]
        return np.sum((st[:, 0, :] - target) ** 2, axis=0) / target.size

    h = 1e-5
    for q in range(p.shape[0]):
        dp = np.zeros_like(p)
        dp[q] = h
        fd = (loss(p + dp) - loss(p - dp)) / (2 * h)
        np.testing.assert_allclose(gp[q], fd, rtol=1e-4, atol=1e-9)
