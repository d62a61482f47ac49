"""Run-axis sharding and the cross-rank reduction, with two gloo ranks on
the CPU (the multi-GPU launch uses the same calls over NCCL)."""

import os

import numpy as np
import pytest


def test_shard_bounds_tile_the_batch():
    from cubie_b200.shard import shard_bounds
    for n in (0, 1, 7, 100, 2 ** 20 + 3):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def test_shard_columns():
    from cubie_b200.shard import shard_columns
    a = np.arange(20).reshape(2, 10)
    b = np.arange(10.0)
    x, y, z = shard_columns([a, b, None], 1, 3)
    assert x.tolist() == [[4, 5, 6], [14, 15, 16]] and y.tolist() == [4.0, 5.0, 6.0] and z is None


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from cubie_b200.shard import aggregate, shard_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lo, hi = shard_bounds(1000, rank, world)
        ms = 10.0 + 5.0 * rank          # rank 1 is the slowest
        solved = float(hi - lo) * 0.5
        out[rank] = aggregate(ms, solved)
    finally:
        dist.destroy_process_group()


def test_aggregate_over_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1] == (15.0, 500.0)


def test_aggregate_without_process_group_is_local():
    from cubie_b200.shard import aggregate
    assert aggregate(3.0, 7.0) == (3.0, 7.0)


def _oracle_solve(inits, params, durations=None):
    """A CPU stand-in for one rank's Solver.solve: the oracle on the rank's
    runs (a SolveResult with the engine's array order)."""
    from cubie_b200.solveresult import SolveResult
    from oracle import OracleSystem, integrate
    osys = OracleSystem(["dx = y", "dy = mu * (1 - x**2) * y - x"], ["x", "y"], ["mu"], {})
    out = integrate(osys, "ros3p", np.asarray(inits), np.asarray(params), float(np.max(durations)),
                    durations=np.asarray(durations), precision=np.float64, rtol=1e-6, atol=1e-6,
                    linear_correction_type="direct", output_types=["state", "iteration_counters"])
    res = SolveResult(state=out["state"], iteration_counters=out["iteration_counters"], status_codes=out["status"])
    res.totals = {"steps": int(out["iteration_counters"][:, 2, :].sum()), "rejections": 0, "newton": 0,
                  "krylov": 0}
    return res


def _split_worker(rank, world, port, out):
    import torch.distributed as dist
    from cubie_b200.shard import distributed_solve
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(3)
        n = 11
        mu = 10 ** rng.uniform(0, 1.5, n)
        x0 = rng.uniform(-2, 2, (2, n))
        res = distributed_solve(_oracle_solve, x0, mu[None, :], {"durations": 2.0 * mu})
        out[rank] = (res.state, res.status_codes, res.totals["steps"])
    finally:
        dist.destroy_process_group()


def test_distributed_solve_splits_and_reassembles_in_order():
    """Two gloo ranks each integrate an interleaved share of a batch (CPU
    stand-in for the per-GPU solve) and both get the whole batch back, equal
    to the unsplit solve, in the caller's run order."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_split_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    rng = np.random.default_rng(3)
    mu = 10 ** rng.uniform(0, 1.5, 11)
    x0 = rng.uniform(-2, 2, (2, 11))
    whole = _oracle_solve(x0, mu[None, :], durations=2.0 * mu)
    for rank in (0, 1):
        state, status, steps = out[rank]
        np.testing.assert_array_equal(state, whole.state)
        np.testing.assert_array_equal(status, whole.status_codes)
        assert steps == whole.totals["steps"]


def test_interleaved_runs_partition_the_batch():
    from cubie_b200.shard import interleaved_runs
    for n, world in ((10, 3), (1, 2), (0, 4), (17, 8)):
        parts = [interleaved_runs(n, r, world) for r in range(world)]
        assert sorted(np.concatenate(parts).tolist()) == list(range(n))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
