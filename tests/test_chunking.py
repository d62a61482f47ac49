"""Run-axis chunk planning and host spill (no GPU): chunk sizes, bounds and
the memory-mapped outputs.  The GPU test that a chunked solve equals the
unchunked one is in ``test_batching_gpu.py``."""

import numpy as np
import pytest

from cubie_b200 import Solver, create_ODE_system
from cubie_b200.chunking import bytes_per_run, host_outputs, output_shapes, plan_chunks


def test_whole_batch_fits_in_one_chunk():
    plan = plan_chunks(10_000, per_run=100, budget=10_000 * 100)
    assert plan.n_chunks == 1 and plan.chunk_runs == 10_000 and plan.bounds() == [(0, 10_000)]


@pytest.mark.parametrize("n,per_run,budget", [(10_000, 100, 200_000), (1_000_003, 64, 10_000_000), (100, 10, 50)])
def test_chunks_fit_two_slots_and_tile_the_runs(n, per_run, budget):
    plan = plan_chunks(n, per_run, budget)
    assert plan.chunk_runs % 32 == 0 and plan.chunk_runs >= 32
    if plan.chunk_runs > 32:
        assert 2 * plan.chunk_runs * per_run <= budget
    b = plan.bounds()
    assert b[0][0] == 0 and b[-1][1] == n and len(b) == plan.n_chunks
    assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))


def test_max_chunk_runs_caps_chunks():
    plan = plan_chunks(5000, per_run=10, budget=10**12, max_chunk_runs=1000)
    assert plan.chunk_runs == 1024 and plan.n_chunks == 5


def test_per_run_footprint_counts_inputs_outputs_and_per_run_arrays():
    sysm = create_ODE_system(["dx = y", "dy = mu * (1 - x**2) * y - x"], states={"x": 2.0, "y": 0.0},
                             parameters={"mu": 10.0}, precision=np.float32)
    solver = Solver(sysm, algorithm="ros3p", save_every=0.5, output_types=["state", "time", "mean"],
                    summarise_every=1.0, sample_summaries_every=0.1)
    prep = solver.prepare(2.0, load=False)
    shapes = output_shapes(solver, prep, 1)
    n_save = prep["n_save"]
    assert shapes["state"][0] == (n_save, 3, 1)
    outputs = sum(int(np.prod(s)) * np.dtype(d).itemsize for s, d in shapes.values())
    assert bytes_per_run(solver, prep) == (2 + 1) * 4 + outputs
    assert bytes_per_run(solver, prep, per_run_arrays=1) == (2 + 1) * 4 + outputs + 8 + 8


def test_host_outputs_spill_to_memory_mapped_files(tmp_path):
    shapes = {"state": ((3, 2, 100), np.dtype(np.float32)), "status": ((100,), np.dtype(np.int32))}
    kept = host_outputs(shapes, spill_threshold=None, spill_dir=str(tmp_path))
    assert all(type(a) is np.ndarray for a in kept.values())
    spilled = host_outputs(shapes, spill_threshold=1000, spill_dir=str(tmp_path))
    assert all(isinstance(a, np.memmap) for a in spilled.values())
    assert spilled["state"].spill_path.startswith(str(tmp_path))
    spilled["state"][...] = 1.5
    assert np.all(np.fromfile(spilled["state"].spill_path, dtype=np.float32) == 1.5)
