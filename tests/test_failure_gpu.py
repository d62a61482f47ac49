"""Failure paths on the GPU, caused on the host: the abort flag polled by
the kernel, non-finite inputs, and the per-run step budget."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]


def _solver(**kw):
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    return Solver(sysm, algorithm="ros3p", rtol=1e-6, atol=1e-6, output_types=["state"], **kw)


def test_abort_flag_stops_every_run(cuda_device):
    import torch
    solver = _solver()
    n = 2048
    rng = np.random.default_rng(0)
    dev = torch.device("cuda", cuda_device)
    prep = solver.prepare(2000.0)
    inits = torch.as_tensor(rng.uniform(-2, 2, (2, n)), device=dev).float()
    params = torch.as_tensor((10 ** rng.uniform(0, 3, n))[None, :], device=dev).float()
    bufs = solver.allocate_outputs(prep, n, dev, torch.float32)
    flag = torch.ones((1,), dtype=torch.int32).pin_memory()     # host memory the kernel polls
    args = solver.make_args(prep, bufs, inits, params, None, n, 2000.0, 0.0, 0.0)
    args.abort_flag = flag.data_ptr()
    prep["module"].launch(args, 1, solver.block_size, 0, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    status = bufs["status"].cpu().numpy()
    assert np.all(status == 32)
    assert int(bufs["totals"][0]) == 0        # checked before the first step of every run


def test_nonfinite_inputs_fail_and_are_masked(cuda_device):
    solver = _solver(max_steps=100_000)
    x0 = np.array([[2.0, np.nan, 1.0], [0.0, 0.0, np.inf]])
    mu = np.array([[10.0, 10.0, 10.0]])
    res = solver.solve(x0, mu, duration=5.0)
    assert res.status_codes[0] == 0
    assert res.status_codes[1] != 0 and res.status_codes[2] != 0
    assert np.all(np.isnan(res.state[..., 1])) and np.all(np.isnan(res.state[..., 2]))
    assert np.all(np.isfinite(res.state[..., 0]))


def test_abort_flag_raised_while_the_launch_runs(cuda_device):
    """The host raises the abort flag while a long persistent launch runs
    (stiff runs with the reference's default minimal-residual stage solves
    take seconds each): the launch ends early, the runs still going end
    with status bit 32, and the runs already finished keep status 0."""
    import time
    import torch
    solver = _solver(max_steps=200_000)
    n = 4096
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", cuda_device)
    mu = 10 ** rng.uniform(0.0, 3.0, n)
    prep = solver.prepare(2000.0, durations=2.0 * mu)
    inits = torch.as_tensor(rng.uniform(-2, 2, (2, n)), device=dev).float()
    params = torch.as_tensor(mu[None, :], device=dev).float()
    durs = torch.as_tensor(2.0 * mu, device=dev, dtype=torch.float64)
    bufs = solver.allocate_outputs(prep, n, dev, torch.float32)
    flag = torch.zeros((1,), dtype=torch.int32).pin_memory()    # host memory the kernel polls
    args = solver.make_args(prep, bufs, inits, params, None, n, 2000.0, 0.0, 0.0, durs)
    args.abort_flag = flag.data_ptr()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    prep["module"].launch(args, 1, solver.block_size, 0, stream.cuda_stream)
    e1.record(stream)
    time.sleep(0.5)
    flag[0] = 1
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    status = bufs["status"].cpu().numpy()
    assert set(np.unique(status).tolist()) <= {0, 32}
    assert np.sum(status == 32) > 0 and np.sum(status == 0) > 0
    assert ms < 10_000.0, ms
