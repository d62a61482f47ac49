"""cbx_solve_noalloc (scratch in a static device array) against cbx_solve.

Both entry points are called through the C ABI on the same inputs and must
give the same outputs, bit for bit, as the persistent and plain kernels do
(``test_persistent_kernel_equals_plain``).  Two calls in a row, on
different inputs, check that the second call does not see the first one's
work counter or totals.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]
N_RUNS = 1000  # not a multiple of the block size


def _inputs(seed):
    rng = np.random.default_rng(seed)
    mu = 10.0 ** rng.uniform(0.0, 2.0, N_RUNS)
    x0 = rng.uniform(-2.0, 2.0, (2, N_RUNS))
    return x0, mu


def test_noalloc_matches_cbx_solve_on_two_calls(cuda_device):
    import torch
    from cubie_b200 import Solver, _native, create_ODE_system

    dev = torch.device("cuda", cuda_device)
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    solver = Solver(sysm, algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type="gmres",
                    preconditioner_type=None, mixed_precision=True, kernel="persistent",
                    output_types=["state", "time", "mean", "max"], save_every=5.0, summarise_every=10.0,
                    device=cuda_device)
    L = _native.lib()
    stream = torch.cuda.current_stream(dev)
    for call, seed in enumerate((11, 12)):
        x0, mu = _inputs(seed)
        duration = 20.0
        prep = solver.prepare(duration)
        inits = torch.as_tensor(x0, device=dev, dtype=torch.float32).contiguous()
        params = torch.as_tensor(mu[None, :], device=dev, dtype=torch.float32).contiguous()

        ref = solver.allocate_outputs(prep, N_RUNS, dev, torch.float32)
        args_ref = solver.make_args(prep, ref, inits, params, None, N_RUNS, duration, 0.0, 0.0)
        prep["module"].launch(args_ref, 1, solver.block_size, 0, stream.cuda_stream)

        out = solver.allocate_outputs(prep, N_RUNS, dev, torch.float32)
        for key in ("state", "state_sum"):
            out[key].fill_(float("nan"))
        out["status"].fill_(-1)
        args = solver.make_args(prep, out, inits, params, None, N_RUNS, duration, 0.0, 0.0)
        args.work_counter = None
        # first call: totals in the scratch array; second: in a caller buffer
        args.totals = None if call == 0 else out["totals"].data_ptr()
        torch.cuda.synchronize(dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = L.cbx_solve_noalloc(prep["module"]._handle, ctypes.byref(args), solver.block_size, 0,
                                 ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.cbx_last_error().decode()
        torch.cuda.synchronize(dev)
        if call == 1:
            # the defining property: after the first call on the device has
            # looked the array up, a call takes no device memory
            assert torch.cuda.mem_get_info(dev)[0] == free_before

        status = out["status"].cpu().numpy()
        np.testing.assert_array_equal(status, ref["status"].cpu().numpy())
        assert np.mean(status == 0) > 0.9
        for key in ("state", "state_sum"):
            np.testing.assert_array_equal(out[key].cpu().numpy(), ref[key].cpu().numpy())
        if call == 1:
            np.testing.assert_array_equal(out["totals"].cpu().numpy(), ref["totals"].cpu().numpy())
            assert int(ref["totals"][0]) > 0


def test_noalloc_rejects_bad_arguments(cuda_device):
    from cubie_b200 import _native
    L = _native.lib()
    assert L.cbx_solve_noalloc(None, None, 128, 0, None) == -1
    assert b"null" in L.cbx_last_error()
