"""Warp-per-system layout on the GPU: a Hodgkin-Huxley cable with a driven
step current, l_stable_dirk_3 + Newton + BiCGSTAB, against the
thread-per-run layout and the oracle (same algorithm, no dense stage
prediction), and the full 64-compartment (256-state) cable."""

import numpy as np
import pytest

from hh_models import hh_cable

pytestmark = pytest.mark.gpu


def _drivers():
    t = np.arange(1000) * 0.05
    return {"driver_sample_period": 0.05, "t0": 0.0, "order": 3, "wrap": False,
            "I": np.where(t < 25.0, 10.0, 0.0)}


def _inputs(nc, n, seed):
    rng = np.random.default_rng(seed)
    _, states, _, _ = hh_cable(nc)
    x0 = np.array(list(states.values()))[:, None] + rng.normal(0, 0.5, (4 * nc, n)) * np.repeat([1.0, 0.01, 0.01, 0.01], nc)[:, None]
    p = np.stack([rng.uniform(80, 160, n), rng.uniform(20, 50, n), rng.uniform(0.1, 1.0, n)])
    return x0, p


def _solver(nc, prec, layout, **kw):
    from cubie_b200 import Solver, create_ODE_system
    eqs, states, params, drivers = hh_cable(nc)
    sysm = create_ODE_system(eqs, states=states, parameters=params, drivers=drivers, precision=prec)
    base = dict(algorithm="l_stable_dirk_3", linear_correction_type="bicgstab", layout=layout,
                attempt_dense_prediction=False, max_steps=200_000)
    base.update(kw)
    return Solver(sysm, **base)


def _tol_units(a, b, atol, rtol):
    return float(np.nanmax(np.abs(a - b) / (atol + rtol * np.abs(b))))


def test_warp_layout_matches_thread_layout_and_oracle(cuda_device):
    from oracle import DriverTable, OracleSystem, integrate
    from cubie_b200.interpolator import ArrayInterpolator
    nc, n, T = 4, 8, 20.0
    kw = dict(rtol=1e-8, atol=1e-8, output_types=["state", "time", "mean", "max"], save_every=2.0,
              summarise_every=10.0, sample_summaries_every=0.5)
    x0, p = _inputs(nc, n, 1)
    warp = _solver(nc, np.float64, "warp", **kw).solve(x0, p, drivers=_drivers(), duration=T,
                                                        nan_error_trajectories=False)
    thread = _solver(nc, np.float64, "thread", **kw).solve(x0, p, drivers=_drivers(), duration=T,
                                                            nan_error_trajectories=False)
    assert warp.status_codes.tolist() == [0] * n
    assert thread.status_codes.tolist() == [0] * n
    assert _tol_units(warp.state, thread.state, 1e-8, 1e-8) < 1.0
    assert _tol_units(warp.state_summaries, thread.state_summaries, 1e-8, 1e-8) < 1.0
    eqs, states, params, drivers = hh_cable(nc)
    osys = OracleSystem(eqs, list(states), list(params), {}, drivers=drivers)
    it = ArrayInterpolator(np.float64, _drivers(), drivers)
    m = it.device_meta()
    osys.driver_table = DriverTable(it.coefficients, it.driver_sample_period, it.t0, it.wrap,
                                    (not it.wrap) and it.boundary_condition == "clamped", np.float64)
    out = integrate(osys, "l_stable_dirk_3", x0, p, T, precision=np.float64, linear_correction_type="bicgstab",
                    save_every=2.0, dense_prediction=False, rtol=1e-8, atol=1e-8)
    assert out["status"].tolist() == [0] * n
    assert _tol_units(warp.state[:, :4 * nc], out["state"][:, :4 * nc], 1e-8, 1e-8) < 1.0


def test_full_cable_warp_layout(cuda_device):
    nc, n, T = 64, 32, 20.0
    x0, p = _inputs(nc, n, 2)
    s = _solver(nc, np.float32, "warp", rtol=1e-5, atol=1e-5, mixed_precision=True,
                output_types=["mean", "max", "peaks[3]"], summarise_every=T, sample_summaries_every=0.1,
                summarise_variables=[f"V{j:02d}" for j in range(nc)])
    r = s.solve(x0, p, drivers=_drivers(), duration=T, nan_error_trajectories=False)
    assert r.status_codes.tolist() == [0] * n
    summ = r.state_summaries
    assert np.all(np.isfinite(summ))
    # per variable: mean, max, 3 peak indices; voltages stay physiological
    # and most driven compartments fire (some conductance draws do not)
    vmean, vmax = summ[0, 0::5, :], summ[0, 1::5, :]
    assert np.all(vmax < 80.0) and np.all(vmean > -100.0) and np.all(vmean < 60.0)
    assert np.mean(vmax[0] > 0.0) > 0.5
    assert r.totals["newton"] > 0 and r.totals["krylov"] > 0


@pytest.mark.parametrize("prec", [np.float64, np.float32])
def test_scratch_placements_agree(cuda_device, prec):
    """The three stage-solve scratch placements ("shared", "local",
    "registers") run the same arithmetic on the 16-compartment cable: same
    statuses, and in FP64 states within a small fraction of the tolerance
    (the compiler may fuse a multiply-add differently in each).  In FP32 at
    rtol 1e-4 such a last-bit difference can move a compartment's spike by
    a fraction of a step, so there the bar is statistical: the median
    state within one tolerance unit, the worst within 100."""
    nc, n, T = 16, 64, 10.0
    x0, p = _inputs(nc, n, 3)
    tol = 1e-8 if prec == np.float64 else 1e-4
    kw = dict(rtol=tol, atol=tol, output_types=["state"], save_every=1.0, dt=0.025,
              mixed_precision=prec == np.float32)
    res = {}
    for place in ("shared", "local", "registers"):
        s = _solver(nc, prec, "warp", scratch_placement=place, **kw)
        res[place] = s.solve(x0, p, drivers=_drivers(), duration=T, nan_error_trajectories=False)
    ref = res["local"]
    assert ref.status_codes.tolist() == [0] * n
    for place in ("shared", "registers"):
        r = res[place]
        assert r.status_codes.tolist() == ref.status_codes.tolist()
        if prec == np.float64:
            assert _tol_units(r.state, ref.state, tol, tol) < 1e-3, place
        else:
            units = np.abs(r.state - ref.state) / (tol + tol * np.abs(ref.state))
            assert float(np.median(units)) < 1.0 and float(np.max(units)) < 100.0, place
