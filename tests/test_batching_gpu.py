"""Batching on the GPU: the heterogeneous launch, the CUDA-graph solve and
the launch-shape autotuner, each against plain Solver.solve results."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]


def test_hetero_launch_matches_separate_solves(cuda_device):
    from test_hetero_emulated import families
    from cubie_b200.hetero import HeteroSolver
    solvers, batches = families()
    hs = HeteroSolver(solvers)
    results = hs.solve(batches, nan_error_trajectories=False)
    # The heterogeneous module and a family's own module are separate
    # compilations of the same loop: the compiler may fuse a multiply-add
    # in one and not the other, and a stiff relaxation run's step sequence
    # amplifies that last bit (a rounding-sized shift of a fast transition
    # moves the state after it by tens of tolerance units), so the bar is
    # statistical rather than bit identity: most runs within 1 tolerance
    # unit, none beyond 100 (the CPU emulation of both, which fuses
    # nothing, agrees bit for bit: test_hetero_emulated.py).
    for s, b, r in zip(solvers, batches, results):
        ref = s.solve(b["initial_values"], b["parameters"], duration=b["duration"], durations=b["durations"],
                      nan_error_trajectories=False)
        assert r.status_codes.tolist() == ref.status_codes.tolist()
        atol, rtol = float(np.max(s.atol)), float(np.max(s.rtol))
        err = np.max(np.abs(r.state.astype(np.float64) - ref.state) / (atol + rtol * np.abs(ref.state)), axis=(0, 1))
        assert float(np.median(err)) < 1.0 and float(np.max(err)) < 100.0, err
        assert abs(r.totals["steps"] - ref.totals["steps"]) <= 0.01 * ref.totals["steps"]


def _vdp_solver(**kw):
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    return Solver(sysm, algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type="gmres",
                  preconditioner_type=None, mixed_precision=True, output_types=["state"], **kw)


def test_graph_solve_matches_solve_on_two_calls(cuda_device):
    solver = _vdp_solver()
    n = 3000
    g = solver.graph(n, 200.0, per_run_durations=True)
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        mu = 10.0 ** rng.uniform(0, 2, n)
        x0 = rng.uniform(-2, 2, (2, n))
        out = g(x0, mu[None, :], 2 * mu)
        ref = solver.solve(x0, mu[None, :], duration=200.0, durations=2 * mu, nan_error_trajectories=False)
        np.testing.assert_array_equal(out["status"].numpy(), ref.status_codes)
        np.testing.assert_array_equal(out["state"].numpy(), ref.state)
        assert int(out["totals"][0]) == ref.totals["steps"]


def test_autotuned_solver_matches_default(cuda_device, tmp_path, monkeypatch):
    monkeypatch.setenv("CUBIE_B200_CACHE_DIR", str(tmp_path))
    rng = np.random.default_rng(3)
    n = 4096
    mu = 10.0 ** rng.uniform(0, 2, n)
    x0 = rng.uniform(-2, 2, (2, n))
    auto = _vdp_solver(block_size="auto")
    r = auto.solve(x0, mu[None, :], duration=200.0, durations=2 * mu, nan_error_trajectories=False)
    assert not auto.autotune_pending and auto.block_size in (32, 64, 128, 256)
    assert len(auto.autotune_result["timings_ms"]) >= 4
    ref = _vdp_solver().solve(x0, mu[None, :], duration=200.0, durations=2 * mu, nan_error_trajectories=False)
    assert r.status_codes.tolist() == ref.status_codes.tolist()
    err = np.abs(r.state - ref.state) / (1e-6 + 1e-6 * np.abs(ref.state))
    assert float(np.max(err)) < 1e-3


@pytest.mark.parametrize("lin", ["gmres", "direct"])
def test_longest_first_claims_leave_results_unchanged(cuda_device, lin):
    """Claiming runs by decreasing horizon (``schedule='auto'`` with per-run
    durations) changes only which lane integrates which run: every run's
    saved state, status and the launch totals equal the index-order ones
    bit for bit."""
    rng = np.random.default_rng(7)
    n = 5000
    mu = 10.0 ** rng.uniform(0, 2.5, n)
    x0 = rng.uniform(-2, 2, (2, n))
    durs = 2.0 * mu
    out = {}
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    # per-run tolerance scales: the claim order then weighs each horizon
    # by its tolerance too
    ts = 10.0 ** rng.uniform(-2, 0, n)
    for sched in ("index", "auto"):
        solver = Solver(sysm, algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type=lin,
                        preconditioner_type=None, mixed_precision=True, output_types=["state"], schedule=sched)
        out[sched] = solver.solve(x0, mu[None, :], duration=float(durs.max()), durations=durs, tol_scale=ts,
                                  nan_error_trajectories=False)
    assert out["auto"].status_codes.tolist() == out["index"].status_codes.tolist()
    np.testing.assert_array_equal(out["auto"].state, out["index"].state)
    assert out["auto"].totals == out["index"].totals


@pytest.mark.parametrize("per_run_horizons", [False, True])
def test_chunked_solve_equals_unchunked(cuda_device, tmp_path, per_run_horizons):
    """A batch forced into five chunks (``max_chunk_runs``), and the same
    with outputs spilled to memory-mapped files, returns exactly what the
    single launch returns: saved states, summaries, counters, statuses and
    the launch totals (regular saves and summaries; or per-run horizons,
    which save the final state only)."""
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    kw = dict(algorithm="ros3p", rtol=1e-6, atol=1e-6, linear_correction_type="direct", mixed_precision=True)
    if per_run_horizons:
        kw["output_types"] = ["state", "iteration_counters"]
    else:
        kw.update(save_every=1.0, summarise_every=2.0, sample_summaries_every=0.5,
                  output_types=["state", "time", "iteration_counters", "mean", "max"])
    rng = np.random.default_rng(11)
    n = 5000
    mu = 10.0 ** rng.uniform(0, 2, n)
    x0 = rng.uniform(-2, 2, (2, n))
    solve_kw = dict(duration=8.0, nan_error_trajectories=False)
    if per_run_horizons:
        solve_kw["durations"] = np.minimum(2.0 * mu, 8.0)
    whole = Solver(sysm, **kw).solve(x0, mu[None, :], **solve_kw)
    chunked_solver = Solver(sysm, max_chunk_runs=1000, **kw)
    chunked = chunked_solver.solve(x0, mu[None, :], **solve_kw)
    assert chunked_solver.chunks == 5
    spill_solver = Solver(sysm, max_chunk_runs=1000, host_spill_threshold=1, spill_dir=str(tmp_path), **kw)
    spilled = spill_solver.solve(x0, mu[None, :], **solve_kw)
    assert isinstance(spilled.state, np.memmap)
    for res in (chunked, spilled):
        assert res.status_codes.tolist() == whole.status_codes.tolist()
        np.testing.assert_array_equal(res.state, whole.state)
        if whole.state_summaries is not None:
            np.testing.assert_array_equal(res.state_summaries, whole.state_summaries)
        np.testing.assert_array_equal(res.iteration_counters, whole.iteration_counters)
        assert res.totals == whole.totals


def test_fp32_floor_routing_matches_separate_solves(cuda_device):
    """An FP32 family with per-run tolerances straddling the FP32 floor (a
    run at rtol 1e-10 among them): the runs below it come back from the FP64
    twin family of the same launch and match an FP64 solve of those runs,
    the others match the FP32 solve, in the caller's order."""
    from test_hetero_emulated import _fp32_vdp_family
    from cubie_b200.hetero import FP32_RTOL_FLOOR, HeteroSolver
    solvers, batches = _fp32_vdp_family()
    ts = np.array([1.0, 1e-3, 1.0, 1e-2, 0.5, 1.0, 1e-4])
    batches[1] = dict(batches[1], tol_scale=ts)
    hs = HeteroSolver(solvers)
    results = hs.solve(batches, nan_error_trajectories=False)
    s, b, r = solvers[1], batches[1], results[1]
    low = 1e-6 * ts < FP32_RTOL_FLOOR
    assert r.state.dtype == np.float64 and r.status_codes.shape == (7,)
    for mask, solver in ((low, s.with_precision(np.float64)), (~low, s)):
        idx = np.where(mask)[0]
        ref = solver.solve(b["initial_values"][:, idx], b["parameters"][:, idx], duration=b["duration"],
                           durations=b["durations"][idx], tol_scale=ts[idx], nan_error_trajectories=False)
        assert r.status_codes[idx].tolist() == ref.status_codes.tolist()
        # separate compilations: the FP32 parity bar (see the test above)
        yr = ref.state.astype(np.float64)
        err = np.abs(r.state[..., idx] - yr) / (1e-6 + 1e-6 * ts[idx] * np.abs(yr))
        assert float(np.max(err)) < 10.0
