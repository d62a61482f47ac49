"""Heterogeneous batch kernel on the CPU (host emulation): three families
of different systems, algorithms and precisions in one launch give exactly
the outputs and iteration totals of solving each family on its own."""

import numpy as np

LOR = ["dx = sigma * (y - x)", "dy = x * (rho - z) - y", "dz = x * y - beta * z"]
VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]
ROB = ["dy1 = -k1 * y1 + k3 * y2 * y3", "dy2 = k1 * y1 - k3 * y2 * y3 - k2 * y2**2", "dy3 = k2 * y2**2"]


def families():
    from cubie_b200 import Solver, create_ODE_system
    rng = np.random.default_rng(1)
    lor = create_ODE_system(LOR, states={"x": 1., "y": 0., "z": 0.}, parameters={"rho": 21.},
                            constants={"sigma": 10., "beta": 8 / 3}, precision=np.float32)
    vdp = create_ODE_system(VDP, states={"x": 2., "y": 0.}, parameters={"mu": 10.}, precision=np.float32)
    rob = create_ODE_system(ROB, states={"y1": 1., "y2": 0., "y3": 0.},
                            parameters={"k1": .04, "k2": 3e7, "k3": 1e4}, precision=np.float64)
    s1 = Solver(lor, algorithm="dormand-prince-54", rtol=1e-6, atol=1e-8, output_types=["state"],
                mixed_precision=True)
    s2 = Solver(vdp, algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type="gmres",
                preconditioner_type=None, output_types=["state"], mixed_precision=True)
    s3 = Solver(rob, algorithm="ros3p", rtol=1e-7, atol=1e-9, output_types=["state"])
    n1, n2, n3 = 5, 7, 4
    b1 = dict(initial_values=rng.uniform(-10, 10, (3, n1)), parameters=rng.uniform(20, 35, (1, n1)),
              duration=2.0, durations=rng.uniform(0.5, 2.0, n1))
    mu = 10 ** rng.uniform(0, 2, n2)
    b2 = dict(initial_values=rng.uniform(-2, 2, (2, n2)), parameters=mu[None, :], duration=float(2 * mu.max()),
              durations=2 * mu)
    kk = np.stack([0.04 * rng.uniform(0.5, 2, n3), 3e7 * rng.uniform(0.5, 2, n3), 1e4 * rng.uniform(0.5, 2, n3)])
    b3 = dict(initial_values=np.tile([[1.], [0.], [0.]], (1, n3)), parameters=kk, duration=100.0,
              durations=rng.uniform(10, 100, n3))
    return [s1, s2, s3], [b1, b2, b3]


def test_hetero_equals_separate_solves():
    from host_emu.emu import run_emulated, run_emulated_hetero
    from cubie_b200.hetero import HeteroSolver
    solvers, batches = families()
    outs = run_emulated_hetero(HeteroSolver(solvers), batches)
    for s, b, o in zip(solvers, batches, outs):
        ref = run_emulated(s, b["initial_values"].astype(s.precision), b["parameters"].astype(s.precision),
                           b["duration"], kernel="persistent", durations=b["durations"])
        assert o["status"].tolist() == ref["status"].tolist()
        np.testing.assert_array_equal(o["state"], ref["state"])
        assert o["totals"].tolist() == ref["totals"].tolist()


def _fp32_vdp_family():
    """The VdP family of ``families`` stepped in FP32 throughout."""
    from cubie_b200 import Solver
    solvers, batches = families()
    s = solvers[1]
    solvers[1] = Solver(s.system, algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type="gmres",
                        preconditioner_type=None, output_types=["state"])
    return solvers, batches


def test_fp32_floor_routes_tight_runs_to_an_fp64_twin():
    """Runs of an FP32 family whose rtol x tol_scale lies below the FP32
    floor go to an FP64 twin family in the same launch; for a
    mixed-precision family only runs below the (lower) mixed floor do (CPU:
    the routing only)."""
    from cubie_b200.hetero import FP32_RTOL_FLOOR, MIXED_RTOL_FLOOR, HeteroSolver
    solvers, batches = _fp32_vdp_family()
    ts = np.array([1.0, 1e-3, 1.0, 1e-2, 0.5, 1.0, 1e-4])     # VdP rtol 1e-6 x scale
    batches[1] = dict(batches[1], tol_scale=ts)
    hs = HeteroSolver(solvers)
    fams, routes = hs.route(batches)
    low = np.where(1e-6 * ts < FP32_RTOL_FLOOR)[0]
    assert low.tolist() == [1, 3, 4, 6]
    assert len(fams) == 4 and len(routes[1]) == 2
    (f_hi, hi), (f_lo, lo) = routes[1]
    assert lo.tolist() == low.tolist() and sorted(hi.tolist() + lo.tolist()) == list(range(7))
    twin, sub = fams[f_lo]
    assert twin.precision == np.float64 and not twin.mixed_precision
    assert twin.algorithm == solvers[1].algorithm and twin.system.state_names == solvers[1].system.state_names
    np.testing.assert_array_equal(sub["initial_values"], batches[1]["initial_values"][:, low])
    np.testing.assert_array_equal(sub["tol_scale"], ts[low])
    # the FP64 family (Robertson) and families without tight runs are untouched
    assert routes[0] == [(0, None)] and routes[2] == [(3, None)]
    assert HeteroSolver(solvers, fp32_floor=None).route(batches)[1][1] == [(1, None)]
    # a mixed-precision family: only the run below the mixed floor (1e-10)
    mixed, mb = families()
    mb[1] = dict(mb[1], tol_scale=ts)
    r = HeteroSolver(mixed).route(mb)[1][1]
    assert [idx.tolist() for _, idx in r] == [[0, 1, 2, 3, 4, 5], [6]] and 1e-6 * 1e-4 < MIXED_RTOL_FLOOR
