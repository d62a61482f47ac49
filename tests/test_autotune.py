"""Launch-shape autotuner: selection, caching and configuration identity
(CPU, with an injected timer)."""

import numpy as np
import pytest

VDP = ["dx = y", "dy = mu * (1 - x**2) * y - x"]


def _solver(**kw):
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    return Solver(sysm, algorithm="ros3p", output_types=["state"], **kw)


def test_choose_picks_fastest_and_skips_failures():
    from cubie_b200.autotune import choose
    assert choose({(128, 1): 5.0, (64, 1): 3.0, (256, 1): float("nan")}) == (64, 1)
    assert choose({(128, 1): 2.0, (64, 1): 2.0}) == (128, 1)
    with pytest.raises(RuntimeError):
        choose({(128, 1): float("nan")})


def test_autotune_uses_timer_and_caches(tmp_path, monkeypatch):
    from cubie_b200.autotune import autotune
    monkeypatch.setenv("CUBIE_B200_CACHE_DIR", str(tmp_path))
    solver = _solver()
    calls = []

    def fake(v):
        calls.append((v.block_size, v.min_blocks_per_sm))
        return {(128, 1): 9.0, (64, 1): 7.5, (256, 1): 8.0, (128, 6): 7.0}[(v.block_size, v.min_blocks_per_sm)]

    cands = [(128, 1), (64, 1), (256, 1), (128, 6)]
    r = autotune(solver, None, None, 2.0, candidates=cands, timer=fake)
    assert (r["block"], r["min_blocks"], r["cached"]) == (128, 6, False)
    assert calls == cands
    r2 = autotune(solver, None, None, 2.0, candidates=cands, timer=fake)
    assert r2["cached"] and (r2["block"], r2["min_blocks"]) == (128, 6)
    assert len(calls) == len(cands)          # served from the cache
    # a different configuration is tuned separately
    other = _solver(rtol=1e-4)
    autotune(other, None, None, 2.0, candidates=cands, timer=fake)
    assert len(calls) == 2 * len(cands)


def test_config_key_ignores_launch_shape():
    from cubie_b200.autotune import config_key, variant
    s = _solver()
    assert config_key(s, 2.0, "gpu") == config_key(variant(s, 256, 3), 2.0, "gpu")
    assert config_key(s, 2.0, "gpu") != config_key(s, 2.0, "other-gpu")


def test_block_size_auto_is_pending_until_first_solve():
    s = _solver(block_size="auto")
    assert s.autotune_pending and s.block_size == 128


def test_warp_layout_tunes_scratch_placement(tmp_path, monkeypatch):
    """With scratch_placement='auto' the warp layout's candidates carry both
    placements; the fastest shape and placement win and are cached."""
    from cubie_b200 import Solver, create_ODE_system
    from cubie_b200.autotune import autotune, default_candidates
    monkeypatch.setenv("CUBIE_B200_CACHE_DIR", str(tmp_path))
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    s = Solver(sysm, algorithm="l_stable_dirk_3", layout="warp", scratch_placement="auto",
               output_types=["state"])
    assert s.placement_pending and s.scratch_placement == "shared"
    cands = default_candidates(s)
    assert {c[2] for c in cands} == {"shared", "local", "registers"} and all(len(c) == 4 for c in cands)
    seen = []

    def fake(v):
        seen.append((v.block_size, v.scratch_placement, v.max_registers))
        return 5.0 if (v.block_size, v.scratch_placement, v.max_registers) == (64, "local", 168) else 9.0

    r = autotune(s, None, None, 2.0, candidates=cands, timer=fake)
    assert (r["block"], r["placement"], r["max_registers"], r["cached"]) == (64, "local", 168, False)
    assert sorted(seen) == sorted((c[0], c[2], c[3]) for c in cands)
    assert autotune(s, None, None, 2.0, candidates=cands, timer=fake)["cached"]
    # the placement is part of the generated source, not of the cache key
    fixed = Solver(sysm, algorithm="l_stable_dirk_3", layout="warp", scratch_placement="local",
                   output_types=["state"])
    assert "SHARED_SCRATCH = false" in fixed.prepare(2.0, load=False)["gen"].source
    assert "SHARED_SCRATCH = true" in s.prepare(2.0, load=False)["gen"].source
    regs = Solver(sysm, algorithm="l_stable_dirk_3", layout="warp", scratch_placement="registers",
                  output_types=["state"])
    src = regs.prepare(2.0, load=False)["gen"].source
    assert "REG_SCRATCH = true" in src and "SHARED_SCRATCH = false" in src
    with pytest.raises(ValueError):
        Solver(sysm, algorithm="l_stable_dirk_3", layout="warp", scratch_placement="texture")


def test_claim_order_weighs_horizon_by_tolerance():
    """Persistent launches claim runs by decreasing estimated work: the
    horizon, times tol_scale^(-1/(q+1)) for an adaptive method of order q
    when per-run tolerance scales are given; fixed steps ignore the scale."""
    import torch
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(VDP, states={"x": 2.0, "y": 0.0}, parameters={"mu": 10.0}, precision=np.float32)
    s = Solver(sysm, algorithm="ros3p", output_types=["state"])      # order 3
    dur = torch.tensor([10.0, 5.0, 1.0], dtype=torch.float64)
    assert s.run_order(dur).tolist() == [0, 1, 2]
    # 5 * (1e-8)^(-1/4) = 500 > 10 * 1 > 1 * (1e-2)^(-1/4) = 3.2
    ts = torch.tensor([1.0, 1e-8, 1e-2], dtype=torch.float64)
    assert s.run_order(dur, ts).tolist() == [1, 0, 2]
    fixed = Solver(sysm, algorithm="l_stable_dirk_3", step_controller="fixed", dt=0.01, output_types=["state"])
    assert fixed.run_order(dur, ts).tolist() == [0, 1, 2]
    assert Solver(sysm, algorithm="ros3p", schedule="index", output_types=["state"]).run_order(dur, ts) is None
