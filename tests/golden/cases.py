"""Seeded parity cases shared by the fixture generator and the tests.

Every case names a system (equation strings), an algorithm alias, the
solver keywords, the integration window and how its seeded inputs are
drawn.  ``make_reference_fixtures.py`` runs each case through the
reference's own kernels (CPU, Numba CUDA simulator) and stores the outputs
as ``ref_<name>.npz``; the tests run the same case through the oracle and
through the CUDA engine.
"""

import numpy as np

LORENZ = dict(
    equations=["dx = sigma * (y - x)", "dy = x * (rho - z) - y", "dz = x * y - beta * z"],
    states=["x", "y", "z"], parameters=["rho"], constants={"sigma": 10.0, "beta": 8.0 / 3.0},
)
VDP = dict(
    equations=["dx = y", "dy = mu * (1 - x**2) * y - x"],
    states=["x", "y"], parameters=["mu"], constants={},
)
DRIVEN = dict(
    equations=["dx = v", "dv = -k * x - c * v + F"],
    states=["x", "v"], parameters=["k", "c"], constants={}, drivers=["F"],
)
FHN = dict(
    equations=["dV = V - V**3 / 3 - w + I", "dw = (V + a - b * w) / tau"],
    states=["V", "w"], parameters=["a", "b", "tau", "I"], constants={},
)


def hh_cable_equations(nc):
    """An nc-compartment Hodgkin-Huxley cable: states V, m, h, n per
    compartment (grouped by variable), parameters gNa, gK, gc, driver I
    injected into compartment 0, sealed ends."""
    V = [f"V{j:02d}" for j in range(nc)]
    eqs = []
    for j in range(nc):
        v, m, h, n = V[j], f"m{j:02d}", f"h{j:02d}", f"n{j:02d}"
        left = V[j - 1] if j > 0 else v
        right = V[j + 1] if j < nc - 1 else v
        inj = "I + " if j == 0 else ""
        eqs.append(f"d{v} = {inj}gc * ({left} - 2 * {v} + {right}) - gNa * {m}**3 * {h} * ({v} - 50.0)"
                   f" - gK * {n}**4 * ({v} + 77.0) - 0.3 * ({v} + 54.4)")
    for j in range(nc):
        v, m = V[j], f"m{j:02d}"
        eqs.append(f"d{m} = 0.1 * ({v} + 40.0) / (1 - exp(-({v} + 40.0) / 10.0)) * (1 - {m})"
                   f" - 4.0 * exp(-({v} + 65.0) / 18.0) * {m}")
    for j in range(nc):
        v, h = V[j], f"h{j:02d}"
        eqs.append(f"d{h} = 0.07 * exp(-({v} + 65.0) / 20.0) * (1 - {h}) - 1.0 / (1 + exp(-({v} + 35.0) / 10.0)) * {h}")
    for j in range(nc):
        v, n = V[j], f"n{j:02d}"
        eqs.append(f"d{n} = 0.01 * ({v} + 55.0) / (1 - exp(-({v} + 55.0) / 10.0)) * (1 - {n})"
                   f" - 0.125 * exp(-({v} + 65.0) / 80.0) * {n}")
    states = [*V, *(f"m{j:02d}" for j in range(nc)), *(f"h{j:02d}" for j in range(nc)),
              *(f"n{j:02d}" for j in range(nc))]
    return dict(equations=eqs, states=states, parameters=["gNa", "gK", "gc"], constants={}, drivers=["I"])


HH64 = hh_cable_equations(64)


def hh_inputs(n, seed, nc=64):
    """Resting cable (V -65, m 0.05, h 0.6, n 0.32) with small seeded
    perturbations; gNa ~ U[80,160], gK ~ U[20,50], gc ~ U[0.1,1]."""
    rng = np.random.default_rng(seed)
    rest = np.repeat([-65.0, 0.05, 0.6, 0.32], nc)[:, None]
    scale = np.repeat([0.5, 0.005, 0.005, 0.005], nc)[:, None]
    x0 = rest + scale * rng.normal(0.0, 1.0, (4 * nc, n))
    p = np.stack([rng.uniform(80, 160, n), rng.uniform(20, 50, n), rng.uniform(0.1, 1.0, n)])
    return x0, p


def vdp_manifold_inputs(x0s, mus):
    """Van der Pol runs started at x0 on y = 0: with x0 slightly above 1 the
    run reaches the fold of the slow manifold within
    mu (x0^2 / 2 - ln x0 - 1/2) time units and makes one fast relaxation
    transition to x ~ -2 early in the window."""
    x0 = np.stack([np.asarray(x0s, dtype=float), np.zeros(len(x0s))])
    return x0, np.asarray(mus, dtype=float)[None, :]


# Constant mass matrices (the reference's ``mass`` argument of
# create_ODE_system): a semi-explicit index-1 DAE (Robertson kinetics with
# its conservation law as the algebraic row, M = diag(1, 1, 0)) and Van der
# Pol with a full, nonsingular M.
ROBER_DAE = dict(
    equations=["dy1 = -k1 * y1 + k3 * y2 * y3", "dy2 = k1 * y1 - k3 * y2 * y3 - k2 * y2**2",
               "dy3 = y1 + y2 + y3 - 1"],
    states=["y1", "y2", "y3"], parameters=["k1", "k2", "k3"], constants={},
    mass=[[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 0.0]],
)
VDP_MASS = dict(VDP, mass=[[2.0, 0.5], [0.5, 1.0]])


def rober_inputs(n, seed):
    rng = np.random.default_rng(seed)
    x0 = np.tile(np.array([[1.0], [0.0], [0.0]]), (1, n))
    p = np.stack([0.04 * rng.uniform(0.5, 2, n), 3e7 * rng.uniform(0.5, 2, n), 1e4 * rng.uniform(0.5, 2, n)])
    return x0, p


def lorenz_inputs(n, seed):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(20.0, 35.0, n)
    x0 = rng.uniform(-10.0, 10.0, (3, n))
    return x0, rho[None, :]


def vdp_inputs(n, seed, mus):
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(-2.0, 2.0, (2, n))
    return x0, np.asarray(mus, dtype=float)[None, :]


def driven_inputs(n, seed):
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(-1.0, 1.0, (2, n))
    p = np.stack([rng.uniform(2.0, 20.0, n), rng.uniform(0.1, 2.0, n)])
    return x0, p


def fhn_inputs(n, seed):
    rng = np.random.default_rng(seed)
    p = np.stack([rng.uniform(0.5, 0.9, n), rng.uniform(0.6, 1.0, n), rng.uniform(8.0, 15.0, n),
                  rng.uniform(0.3, 0.6, n)])
    x0 = np.stack([rng.uniform(-1.0, 1.0, n), rng.uniform(-0.5, 0.5, n)])
    return x0, p


CASES = {
    "lorenz_dp54_f32": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float32",
                            inputs=("lorenz", 8, 1), duration=1.0,
                            kwargs=dict(rtol=1e-6, atol=1e-8, save_every=0.05, summarise_every=0.25,
                                        sample_summaries_every=0.05,
                                        output_types=["state", "time", "iteration_counters", "mean", "max"])),
    "lorenz_dp54_f64": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float64",
                            inputs=("lorenz", 8, 1), duration=1.0,
                            kwargs=dict(rtol=1e-8, atol=1e-10, save_every=0.05, summarise_every=0.25,
                                        sample_summaries_every=0.05,
                                        output_types=["state", "time", "iteration_counters", "mean", "max"])),
    "lorenz_dp54_pid_f64": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float64",
                                inputs=("lorenz", 4, 2), duration=0.5,
                                kwargs=dict(rtol=1e-7, atol=1e-9, save_every=0.1, step_controller="pid",
                                            kp=0.7, ki=-0.4, kd=0.1, output_types=["state", "time"])),
    "lorenz_dp54_i_f64": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float64",
                              inputs=("lorenz", 4, 3), duration=0.5,
                              kwargs=dict(rtol=1e-7, atol=1e-9, save_every=0.1, step_controller="i",
                                          output_types=["state", "time"])),
    "lorenz_dp54_gus_f64": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float64",
                                inputs=("lorenz", 4, 4), duration=0.5,
                                kwargs=dict(rtol=1e-7, atol=1e-9, save_every=0.1, step_controller="gustafsson",
                                            output_types=["state", "time"])),
    "vdp_ros3p_f32": dict(system=VDP, algorithm="ros3p", precision="float32",
                          inputs=("vdp", 4, 5, [1.0, 3.0, 10.0, 30.0]), duration=2.0,
                          kwargs=dict(rtol=1e-6, atol=1e-6, save_every=0.25,
                                      output_types=["state", "time", "iteration_counters"])),
    "vdp_ros3p_bicgstab_f64": dict(system=VDP, algorithm="ros3p", precision="float64",
                                   inputs=("vdp", 4, 6, [1.0, 3.0, 10.0, 30.0]), duration=2.0,
                                   kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.25,
                                               linear_correction_type="bicgstab",
                                               output_types=["state", "time", "iteration_counters"])),
    "vdp_radau_f32": dict(system=VDP, algorithm="radau", precision="float32",
                          inputs=("vdp", 2, 7, [2.0, 20.0]), duration=0.5,
                          kwargs=dict(rtol=1e-6, atol=1e-6, save_every=0.125,
                                      output_types=["state", "time", "iteration_counters"])),
    "vdp_radau_f64": dict(system=VDP, algorithm="radau", precision="float64",
                          inputs=("vdp", 2, 8, [2.0, 20.0]), duration=0.5,
                          kwargs=dict(rtol=1e-8, atol=1e-8, save_every=0.125,
                                      output_types=["state", "time", "iteration_counters"])),
    "vdp_dirk3_bicgstab_f32": dict(system=VDP, algorithm="l_stable_dirk_3", precision="float32",
                                   inputs=("vdp", 2, 9, [2.0, 10.0]), duration=0.5,
                                   kwargs=dict(dt=0.01, rtol=1e-6, atol=1e-6, save_every=0.125,
                                               linear_correction_type="bicgstab",
                                               output_types=["state", "time", "iteration_counters"])),
    "vdp_sdirk4_f64": dict(system=VDP, algorithm="l_stable_sdirk_4", precision="float64",
                           inputs=("vdp", 2, 10, [2.0, 10.0]), duration=0.5,
                           kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.125,
                                       output_types=["state", "time", "iteration_counters"])),
    "fhn_dp54_peaks_f32": dict(system=FHN, algorithm="dormand-prince-54", precision="float32",
                               inputs=("fhn", 4, 11), duration=40.0,
                               kwargs=dict(rtol=1e-6, atol=1e-6, save_every=1.0, summarise_every=20.0,
                                           sample_summaries_every=0.5,
                                           output_types=["state", "time", "peaks[3]", "std", "rms", "min"])),
    "driven_dp54_clamped_f64": dict(system=DRIVEN, algorithm="dormand-prince-54", precision="float64",
                                    inputs=("driven", 4, 13), duration=3.0,
                                    drivers=dict(seed=21, n_samples=16, period=0.2, t0=0.1, order=3, wrap=False,
                                                 boundary_condition="clamped"),
                                    kwargs=dict(rtol=1e-8, atol=1e-8, save_every=0.25,
                                                output_types=["state", "time"])),
    "driven_dp54_periodic_f32": dict(system=DRIVEN, algorithm="dormand-prince-54", precision="float32",
                                     inputs=("driven", 4, 14), duration=4.0,
                                     drivers=dict(seed=22, n_samples=11, period=0.3, t0=0.0, order=3, wrap=True,
                                                  boundary_condition="periodic"),
                                     kwargs=dict(rtol=1e-6, atol=1e-6, save_every=0.5,
                                                 output_types=["state", "time"])),
    "driven_ros3p_clamped_f64": dict(system=DRIVEN, algorithm="ros3p", precision="float64",
                                     inputs=("driven", 4, 15), duration=3.0,
                                     drivers=dict(seed=23, n_samples=16, period=0.2, t0=0.1, order=3, wrap=False,
                                                  boundary_condition="clamped"),
                                     kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.25,
                                                 output_types=["state", "time", "iteration_counters"])),
    "lorenz_step_too_small_f32": dict(system=LORENZ, algorithm="dormand-prince-54", precision="float32",
                                      inputs=("lorenz", 2, 12), duration=1.0,
                                      kwargs=dict(rtol=1e-12, atol=1e-14, dt=0.01, dt_min=0.005, dt_max=0.1,
                                                  output_types=["state", "time"])),
}

# One case per further algorithm of the reference's registries and its
# single-purpose steps (explicit/backward Euler, predictor-corrector,
# Crank-Nicolson): short windows so the simulator finishes in seconds.
_FIX = ["state", "time"]
_ITS = ["state", "time", "iteration_counters"]
_VDP2 = ("vdp", 2, 40, [2.0, 10.0])
CASES.update({
    "lorenz_euler_f64": dict(system=LORENZ, algorithm="euler", precision="float64", inputs=("lorenz", 4, 31),
                             duration=0.2, kwargs=dict(dt=1e-3, rtol=1e-6, atol=1e-6, save_every=0.05,
                                                       output_types=_FIX)),
    "lorenz_ralston_f32": dict(system=LORENZ, algorithm="ralston-33", precision="float32", inputs=("lorenz", 4, 32),
                               duration=0.2, kwargs=dict(dt=2e-3, rtol=1e-5, atol=1e-5, save_every=0.05,
                                                         output_types=_FIX)),
    "lorenz_rk4_f64": dict(system=LORENZ, algorithm="classical-rk4", precision="float64", inputs=("lorenz", 4, 33),
                           duration=0.2, kwargs=dict(dt=2e-3, rtol=1e-6, atol=1e-6, save_every=0.05,
                                                     output_types=_FIX)),
    "lorenz_bs32_f64": dict(system=LORENZ, algorithm="bogacki-shampine-32", precision="float64",
                            inputs=("lorenz", 4, 34), duration=0.5,
                            kwargs=dict(rtol=1e-7, atol=1e-9, save_every=0.1, output_types=_ITS)),
    "lorenz_cashkarp_f64": dict(system=LORENZ, algorithm="cash-karp-54", precision="float64",
                                inputs=("lorenz", 4, 35), duration=0.5,
                                kwargs=dict(rtol=1e-8, atol=1e-10, save_every=0.1, output_types=_ITS)),
    "lorenz_fehlberg_f64": dict(system=LORENZ, algorithm="fehlberg-45", precision="float64",
                                inputs=("lorenz", 4, 36), duration=0.5,
                                kwargs=dict(rtol=1e-8, atol=1e-10, save_every=0.1, output_types=_ITS)),
    "lorenz_tsit5_f64": dict(system=LORENZ, algorithm="tsit5", precision="float64", inputs=("lorenz", 4, 37),
                             duration=0.5, kwargs=dict(rtol=1e-8, atol=1e-10, save_every=0.1, output_types=_ITS)),
    "lorenz_vern7_f64": dict(system=LORENZ, algorithm="vern7", precision="float64", inputs=("lorenz", 4, 38),
                             duration=0.5, kwargs=dict(rtol=1e-9, atol=1e-11, save_every=0.1, output_types=_ITS)),
    "lorenz_dop853_f64": dict(system=LORENZ, algorithm="dop853", precision="float64", inputs=("lorenz", 4, 39),
                              duration=0.5, kwargs=dict(rtol=1e-9, atol=1e-11, save_every=0.1, output_types=_ITS)),
    "vdp_be_f64": dict(system=VDP, algorithm="backwards_euler", precision="float64", inputs=_VDP2, duration=0.5,
                       kwargs=dict(dt=0.01, rtol=1e-6, atol=1e-6, save_every=0.125, output_types=_ITS)),
    "vdp_bepc_f32": dict(system=VDP, algorithm="backwards_euler_pc", precision="float32",
                         inputs=("vdp", 2, 41, [2.0, 10.0]), duration=0.5,
                         kwargs=dict(dt=0.01, rtol=1e-6, atol=1e-6, save_every=0.125, output_types=_ITS)),
    "vdp_cn_f64": dict(system=VDP, algorithm="crank_nicolson", precision="float64", inputs=("vdp", 2, 42, [2.0, 10.0]),
                       duration=0.5, kwargs=dict(rtol=1e-6, atol=1e-6, save_every=0.125, output_types=_ITS)),
    "vdp_trap_f32": dict(system=VDP, algorithm="trapezoidal_dirk", precision="float32",
                         inputs=("vdp", 2, 43, [2.0, 10.0]), duration=0.5,
                         kwargs=dict(dt=0.01, rtol=1e-6, atol=1e-6, save_every=0.125, output_types=_ITS)),
    "vdp_sdirk22_f64": dict(system=VDP, algorithm="sdirk_2_2", precision="float64",
                            inputs=("vdp", 2, 44, [2.0, 10.0]), duration=0.5,
                            kwargs=dict(dt=0.01, rtol=1e-7, atol=1e-7, save_every=0.125, output_types=_ITS)),
    "vdp_midpoint_f64": dict(system=VDP, algorithm="implicit_midpoint", precision="float64",
                             inputs=("vdp", 2, 45, [2.0, 10.0]), duration=0.5,
                             kwargs=dict(dt=0.01, rtol=1e-7, atol=1e-7, save_every=0.125, output_types=_ITS)),
    "vdp_kvaerno3_f64": dict(system=VDP, algorithm="kvaerno3", precision="float64",
                             inputs=("vdp", 2, 46, [2.0, 10.0]), duration=0.5,
                             kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.125, output_types=_ITS)),
    "vdp_kvaerno5_f32": dict(system=VDP, algorithm="kvaerno5", precision="float32",
                             inputs=("vdp", 2, 47, [2.0, 10.0]), duration=0.5,
                             kwargs=dict(rtol=1e-5, atol=1e-5, save_every=0.125, output_types=_ITS)),
    "vdp_gl2_f32": dict(system=VDP, algorithm="firk_gauss_legendre_2", precision="float32",
                        inputs=("vdp", 2, 48, [2.0, 10.0]), duration=0.5,
                        kwargs=dict(dt=0.02, rtol=1e-6, atol=1e-6, save_every=0.125, output_types=_ITS)),
    "vdp_gl4_f64": dict(system=VDP, algorithm="firk_gauss_legendre_4", precision="float64",
                        inputs=("vdp", 2, 49, [2.0, 10.0]), duration=0.5,
                        kwargs=dict(dt=0.025, rtol=1e-8, atol=1e-8, save_every=0.125, output_types=_ITS)),
    "vdp_rodas3p_f64": dict(system=VDP, algorithm="rodas3p", precision="float64",
                            inputs=("vdp", 4, 50, [1.0, 3.0, 10.0, 30.0]), duration=1.0,
                            kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.25, output_types=_ITS)),
    "fhn_dp54_derivs_f64": dict(system=FHN, algorithm="dormand-prince-54", precision="float64",
                                inputs=("fhn", 4, 52), duration=30.0,
                                kwargs=dict(rtol=1e-8, atol=1e-8, save_every=1.0, summarise_every=10.0,
                                            sample_summaries_every=0.25,
                                            output_types=["state", "time", "dxdt_max", "dxdt_min",
                                                          "d2xdt2_max"])),
    "fhn_dp54_derivs_f32": dict(system=FHN, algorithm="dormand-prince-54", precision="float32",
                                inputs=("fhn", 4, 53), duration=30.0,
                                kwargs=dict(rtol=1e-6, atol=1e-6, save_every=1.0, summarise_every=10.0,
                                            sample_summaries_every=0.25,
                                            output_types=["state", "time", "mean", "dxdt_min", "d2xdt2_max",
                                                          "d2xdt2_min"])),
    "vdp_rosenbrock23_f32": dict(system=VDP, algorithm="rosenbrock23", precision="float32",
                                 inputs=("vdp", 4, 51, [1.0, 3.0, 10.0, 30.0]), duration=1.0,
                                 kwargs=dict(rtol=1e-5, atol=1e-5, save_every=0.25, output_types=_ITS)),
})


# Stiff Van der Pol at the headline's stiffness (mu up to 1000) over a
# window with one relaxation transition per run, and the 64-compartment
# (256-state) Hodgkin-Huxley cable with its step current over a window that
# holds the first spike.  ``engine`` holds settings of this engine only
# (the fixture generator does not pass them to the reference).
# ``counters_rounding_sensitive`` marks a case whose step and iteration
# counts follow last-bit differences (BiCGSTAB on a singular-mass stage
# system): compared in tolerance units, not counter by counter.
# ``slow_oracle`` marks cases that take the NumPy oracle minutes (tens of
# thousands of FP32 Krylov iterations per stiff run; the 256-state cable's
# dense Jacobians): their oracle pins run when CBX_SLOW_PINS=1, and
# the GPU tests compare them with the reference fixture only.
_MU = ("vdp_manifold", [1.4, 1.2, 1.1], [100.0, 300.0, 1000.0])
_HH_DRV = dict(seed=0, n_samples=1000, period=0.01, t0=0.0, order=3, wrap=False, boundary_condition="clamped",
               step=(10.0, 5.0))
CASES.update({
    "vdp_stiff_ros3p_f32": dict(system=VDP, algorithm="ros3p", precision="float32", inputs=_MU, duration=20.0,
                                slow_oracle=True,
                                kwargs=dict(rtol=1e-6, atol=1e-6, save_every=2.0, output_types=_ITS)),
    "vdp_stiff_ros3p_f64": dict(system=VDP, algorithm="ros3p", precision="float64", inputs=_MU, duration=20.0,
                                kwargs=dict(rtol=1e-6, atol=1e-6, save_every=2.0, linear_correction_type="bicgstab",
                                            output_types=_ITS)),
    "vdp_stiff_radau_f32": dict(system=VDP, algorithm="radau", precision="float32", inputs=_MU, duration=20.0,
                                slow_oracle=True,
                                kwargs=dict(rtol=1e-6, atol=1e-6, save_every=2.0, linear_correction_type="bicgstab",
                                            output_types=_ITS)),
    "vdp_stiff_radau_f64": dict(system=VDP, algorithm="radau", precision="float64", inputs=_MU, duration=20.0,
                                kwargs=dict(rtol=1e-6, atol=1e-6, save_every=2.0, linear_correction_type="bicgstab",
                                            output_types=_ITS)),
    "hh64_dirk3_bicgstab_f32": dict(system=HH64, algorithm="l_stable_dirk_3", precision="float32",
                                    inputs=("hh", 2, 60), duration=4.0, drivers=_HH_DRV, slow_oracle=True,
                                    engine=dict(layout="warp"),
                                    kwargs=dict(dt=0.025, rtol=1e-4, atol=1e-4, linear_correction_type="bicgstab",
                                                save_every=0.5, summarise_every=4.0, sample_summaries_every=0.05,
                                                summarise_variables=[f"V{j:02d}" for j in range(64)],
                                                saved_state_indices=list(range(64)),
                                                output_types=["state", "time", "iteration_counters", "mean",
                                                              "max"])),
})


CASES.update({
    "rober_dae_radau_f64": dict(system=ROBER_DAE, algorithm="radau", precision="float64", inputs=("rober", 3, 70),
                                counters_rounding_sensitive=True,
                                duration=1.0, kwargs=dict(rtol=1e-6, atol=1e-8, save_every=0.25,
                                                          linear_correction_type="bicgstab", output_types=_ITS)),
    "rober_dae_dirk3_f64": dict(system=ROBER_DAE, algorithm="l_stable_dirk_3", precision="float64",
                                inputs=("rober", 3, 71), duration=0.5,
                                kwargs=dict(dt=1e-3, rtol=1e-6, atol=1e-8, save_every=0.125,
                                            linear_correction_type="bicgstab", output_types=_ITS)),
    "vdp_mass_radau_f32": dict(system=VDP_MASS, algorithm="radau", precision="float32",
                               inputs=("vdp", 3, 74, [1.0, 3.0, 10.0]), duration=2.0,
                               kwargs=dict(rtol=1e-6, atol=1e-6, save_every=0.5, output_types=_ITS)),
})


def case_inputs(case):
    kind = case["inputs"][0]
    if kind == "lorenz":
        return lorenz_inputs(case["inputs"][1], case["inputs"][2])
    if kind == "vdp":
        return vdp_inputs(case["inputs"][1], case["inputs"][2], case["inputs"][3])
    if kind == "fhn":
        return fhn_inputs(case["inputs"][1], case["inputs"][2])
    if kind == "driven":
        return driven_inputs(case["inputs"][1], case["inputs"][2])
    if kind == "hh":
        return hh_inputs(case["inputs"][1], case["inputs"][2])
    if kind == "rober":
        return rober_inputs(case["inputs"][1], case["inputs"][2])
    if kind == "vdp_manifold":
        return vdp_manifold_inputs(case["inputs"][1], case["inputs"][2])
    raise KeyError(kind)


def case_drivers(case):
    """The drivers dictionary of a case (reference ``solve(drivers=...)``
    format), or None."""
    spec = case.get("drivers")
    if spec is None:
        return None
    rng = np.random.default_rng(spec["seed"])
    out = {"driver_sample_period": spec["period"], "t0": spec["t0"], "order": spec["order"],
           "wrap": spec["wrap"], "boundary_condition": spec["boundary_condition"]}
    if spec.get("step") is not None:
        # a step current: ``level`` before ``t_off``, 0 after
        level, t_off = spec["step"]
        t = spec["t0"] + spec["period"] * np.arange(spec["n_samples"])
        for name in case["system"]["drivers"]:
            out[name] = np.where(t < t_off, level, 0.0)
        return out
    for name in case["system"]["drivers"]:
        samples = rng.uniform(-1.0, 1.0, spec["n_samples"])
        if spec["boundary_condition"] == "periodic":
            samples[-1] = samples[0]
        out[name] = samples
    return out
