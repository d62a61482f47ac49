"""Discrete adjoint on the GPU against the FP64 forward-sensitivity
reference (oracle/sensitivity.py), through the torch autograd wrapper."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FHN = ["dV = V - V**3 / 3 - w + I", "dw = (V + a - b * w) / tau"]
VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]


def fhn_case(n, seed):
    rng = np.random.default_rng(seed)
    p = np.stack([rng.uniform(0.5, 0.9, n), rng.uniform(0.6, 1.0, n), rng.uniform(8.0, 15.0, n),
                  rng.uniform(0.3, 0.6, n)])
    x0 = np.stack([rng.uniform(-1.0, 1.0, n), rng.uniform(-0.5, 0.5, n)])
    return x0, p, rng


def vdp_case(n, seed):
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(-2.0, 2.0, (2, n))
    mu = 10.0 ** rng.uniform(0.0, 1.0, n)
    return x0, mu[None, :], rng


def _solver(eqs, states, params, prec, **kw):
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(eqs, states={s: 0.0 for s in states}, parameters={q: 1.0 for q in params},
                             precision=prec)
    return Solver(sysm, output_types=["state"], save_every=1.0, adjoint=True, **kw)


def _torch_grads(solver, x0, p, T, target, **kw):
    import torch
    from cubie_b200.adjoint import solve_ivp_adjoint
    dt = torch.float64 if solver.precision == np.float64 else torch.float32
    xi = torch.tensor(x0, device="cuda", dtype=dt, requires_grad=True)
    pi = torch.tensor(p, device="cuda", dtype=dt, requires_grad=True)
    state, status = solve_ivp_adjoint(solver, xi, pi, T, **kw)
    tgt = torch.tensor(target, device="cuda", dtype=dt)
    loss = torch.mean((state[:, 0, :] - tgt) ** 2)
    loss.backward()
    g_rows = np.zeros(tuple(state.shape))
    g_rows[:, 0, :] = 2.0 * (state[:, 0, :].detach().double().cpu().numpy() - target) / target.size
    return (state.detach().cpu().numpy(), status.cpu().numpy(), xi.grad.cpu().numpy(), pi.grad.cpu().numpy(),
            g_rows)


def _reference(eqs, states, params, x0, p, T, g_rows):
    from oracle.sensitivity import SensitivitySystem, trajectory_gradients
    ssys = SensitivitySystem(eqs, states, params)
    return trajectory_gradients(ssys, x0, p, np.arange(int(T) + 1, dtype=float), g_rows)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("prec,rtol,mixed,bound", [(np.float64, 1e-10, False, 1e-7),
                                                   (np.float32, 1e-6, True, 2e-3)])
def test_erk_adjoint_matches_forward_sensitivities(cuda_device, prec, rtol, mixed, bound):
    x0, p, rng = fhn_case(64, 3)
    T = 20.0
    target = rng.uniform(-1.0, 1.0, (int(T) + 1, 64))
    solver = _solver(FHN, ["V", "w"], ["a", "b", "tau", "I"], prec, algorithm="dormand-prince-54",
                     rtol=rtol, atol=rtol, mixed_precision=mixed)
    state, status, gi, gp, g_rows = _torch_grads(solver, x0, p, T, target)
    assert np.all(status == 0)
    ref_state, gy0, gpr = _reference(FHN, ["V", "w"], ["a", "b", "tau", "I"], x0, p, T, g_rows)
    assert _rel(gi, gy0) < bound
    assert _rel(gp, gpr) < bound


@pytest.mark.parametrize("lin", ["gmres", "minimal_residual"])
def test_rosenbrock_adjoint_matches_forward_sensitivities(cuda_device, lin):
    x0, p, rng = vdp_case(32, 4)
    T = 10.0
    target = rng.uniform(-1.0, 1.0, (int(T) + 1, 32))
    kw = dict(preconditioner_type=None) if lin == "gmres" else {}
    solver = _solver(VDP, ["x", "y"], ["mu"], np.float64, algorithm="ros3p", rtol=1e-9, atol=1e-9,
                     linear_correction_type=lin, **kw)
    state, status, gi, gp, g_rows = _torch_grads(solver, x0, p, T, target, max_ckpts=4096)
    assert np.all(status == 0)
    ref_state, gy0, gpr = _reference(VDP, ["x", "y"], ["mu"], x0, p, T, g_rows)
    assert _rel(gi, gy0) < 1e-5
    assert _rel(gp, gpr) < 1e-5


@pytest.mark.parametrize("mixed", [False, True])
def test_adjoint_is_independent_of_checkpoint_spacing(cuda_device, mixed):
    """Every spacing replays the forward's steps exactly (spacing 1 restarts
    from a stored state at every step), so the gradients agree bit for bit;
    the mixed-precision case covers the compensated state update."""
    import torch
    from cubie_b200.adjoint import AdjointIntegrator
    x0, p, rng = fhn_case(100, 5)
    solver = _solver(FHN, ["V", "w"], ["a", "b", "tau", "I"], np.float32, algorithm="dormand-prince-54",
                     rtol=1e-6, atol=1e-6, mixed_precision=mixed)
    xi = torch.tensor(x0, device="cuda", dtype=torch.float32)
    pi = torch.tensor(p, device="cuda", dtype=torch.float32)
    out = []
    for every, cap in ((64, 64), (3, 4000), (1, 4000)):
        integ = AdjointIntegrator(solver, ckpt_every=every, max_ckpts=cap)
        state, status, saved = integ.forward(xi, pi, 20.0)
        g = torch.ones_like(state)
        out.append([t.cpu().numpy() for t in integ.backward(saved, g)] + [state.cpu().numpy(), status.cpu().numpy()])
    for other in out[1:]:
        for a, b in zip(out[0], other):
            np.testing.assert_array_equal(a, b)


def test_adjoint_forward_outputs_equal_solve(cuda_device):
    import torch
    from cubie_b200.adjoint import AdjointIntegrator
    x0, p, _ = fhn_case(300, 6)
    solver = _solver(FHN, ["V", "w"], ["a", "b", "tau", "I"], np.float32, algorithm="dormand-prince-54",
                     rtol=1e-6, atol=1e-6, mixed_precision=True)
    res = solver.solve(x0, p, duration=30.0, nan_error_trajectories=False)
    integ = AdjointIntegrator(solver)
    state, status, _ = integ.forward(torch.tensor(x0, device="cuda", dtype=torch.float32),
                                     torch.tensor(p, device="cuda", dtype=torch.float32), 30.0)
    np.testing.assert_array_equal(state.cpu().numpy(), res.state)
    np.testing.assert_array_equal(status.cpu().numpy(), res.status_codes)


def test_checkpoint_capacity_exhaustion_sets_status_32(cuda_device):
    import torch
    from cubie_b200.adjoint import AdjointIntegrator
    x0, p, _ = fhn_case(8, 7)
    solver = _solver(FHN, ["V", "w"], ["a", "b", "tau", "I"], np.float64, algorithm="dormand-prince-54",
                     rtol=1e-10, atol=1e-10)
    integ = AdjointIntegrator(solver, ckpt_every=2, max_ckpts=3)
    state, status, _ = integ.forward(torch.tensor(x0, device="cuda"), torch.tensor(p, device="cuda"), 20.0)
    assert np.all(status.cpu().numpy() == 32)


LORENZ = ["dx = sigma * (y - x)", "dy = x * (rho - z) - y", "dz = x * y - beta * z"]


def test_lorenz_adjoint_with_per_run_tolerances(cuda_device):
    """The adjoint of the mixed three-system batch's Lorenz family: DP54 with
    FP32 stepping and FP64 control, per-run tolerance scales (rtol from 1e-7
    to 1e-5, as the batch draws them), loss = mean squared error of every
    saved state over a bounded window (t in [0, 2], saved every 0.25)
    against seeded targets.  Gradients with respect to the initial states
    and rho against the FP64 forward sensitivities."""
    import torch
    from cubie_b200 import Solver, create_ODE_system
    from cubie_b200.adjoint import AdjointIntegrator
    from oracle.sensitivity import SensitivitySystem, trajectory_gradients
    n, T, every = 16, 2.0, 0.25
    rng = np.random.default_rng(21)
    rho = rng.uniform(20.0, 35.0, n)
    x0 = rng.uniform(-10.0, 10.0, (3, n))
    ts = 10.0 ** rng.uniform(-2.0, 0.0, n)
    rows = int(round(T / every)) + 1
    target = rng.uniform(-10.0, 10.0, (rows, 3, n))
    consts = {"sigma": 10.0, "beta": 8.0 / 3.0}
    sysm = create_ODE_system(LORENZ, states={"x": 1.0, "y": 0.0, "z": 0.0}, parameters={"rho": 21.0},
                             constants=consts, precision=np.float32)
    solver = Solver(sysm, algorithm="dormand-prince-54", rtol=1e-5, atol=1e-7, output_types=["state"],
                    save_every=every, mixed_precision=True, adjoint=True)
    integ = AdjointIntegrator(solver, ckpt_every=64, max_ckpts=64)
    xi = torch.tensor(x0, device="cuda", dtype=torch.float32)
    pi = torch.tensor(rho[None, :], device="cuda", dtype=torch.float32)
    state, status, saved = integ.forward(xi, pi, T, tol_scale=ts)
    assert status.cpu().numpy().tolist() == [0] * n
    s_np = state.double().cpu().numpy()
    g_rows = 2.0 * (s_np - target) / target.size
    gi, gp = integ.backward(saved, torch.tensor(g_rows, device="cuda", dtype=torch.float32))
    ssys = SensitivitySystem(LORENZ, ["x", "y", "z"], ["rho"], consts)
    _, gy0, gpr = trajectory_gradients(ssys, x0, rho[None, :], np.arange(rows) * every, g_rows,
                                       rtol=1e-11, atol=1e-11)
    assert _rel(gi.double().cpu().numpy(), gy0) < 5e-3
    assert _rel(gp.double().cpu().numpy(), gpr) < 5e-3
