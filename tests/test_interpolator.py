"""Array drivers: coefficients and evaluation against the reference's own
``ArrayInterpolator`` (fixture ``golden/ref_interpolator.npz`` made by
``golden/make_interpolator_fixture.py``), plus its input validation."""

from pathlib import Path

import numpy as np
import pytest

from cubie_b200.interpolator import ArrayInterpolator

GOLDEN = Path(__file__).resolve().parent / "golden"
CONFIGS = [
    ("cubic_clamped_f32", 3, False, "clamped", 2, "float32"),
    ("cubic_clamped_f64", 3, False, "clamped", 2, "float64"),
    ("cubic_periodic_f64", 3, True, "periodic", 1, "float64"),
    ("cubic_natural_f64", 3, False, "natural", 2, "float64"),
    ("cubic_notaknot_f64", 3, False, "not-a-knot", 1, "float64"),
    ("quadratic_clamped_f64", 2, False, "clamped", 1, "float64"),
    ("quintic_natural_f64", 5, False, "natural", 1, "float64"),
    ("linear_clamped_f32", 1, False, "clamped", 1, "float32"),
]


@pytest.mark.parametrize("name,order,wrap,bc,ni,prec", CONFIGS)
def test_matches_reference_interpolator(name, order, wrap, bc, ni, prec):
    ref = np.load(GOLDEN / "ref_interpolator.npz")
    samples = ref[name + "__samples"]
    d = {"driver_sample_period": 0.25, "t0": 0.5, "order": order, "wrap": wrap, "boundary_condition": bc}
    for k in range(ni):
        d[f"d{k}"] = samples[:, k]
    p = np.dtype(prec).type
    interp = ArrayInterpolator(p, d, [f"d{k}" for k in range(ni)])
    rc = ref[name + "__coefficients"]
    assert interp.coefficients.shape == rc.shape
    scale = max(1.0, float(np.max(np.abs(rc))))
    tol = 1e-12 if prec == "float64" else 2e-6
    assert np.max(np.abs(interp.coefficients - rc)) <= tol * scale
    vals = interp.evaluate(ref[name + "__query"].astype(p))
    assert np.max(np.abs(vals - ref[name + "__values"].reshape(vals.shape))) <= tol * scale


def test_derivative_matches_finite_difference():
    rng = np.random.default_rng(3)
    d = {"driver_sample_period": 0.1, "t0": 0.0, "order": 3, "wrap": False, "F": rng.uniform(-1, 1, 20)}
    interp = ArrayInterpolator(np.float64, d, ["F"])
    t = np.linspace(0.05, 1.8, 37)
    h = 1e-6
    fd = (interp.evaluate(t + h) - interp.evaluate(t - h)) / (2 * h)
    np.testing.assert_allclose(interp.evaluate(t, derivative=True), fd, rtol=1e-5, atol=1e-6)


def test_defaults_and_padding():
    d = {"time": np.arange(6) * 0.5, "F": np.arange(6.0)}
    clamped = ArrayInterpolator(np.float64, dict(d, wrap=False), ["F"])
    assert clamped.boundary_condition == "clamped" and clamped.num_segments == 7
    meta = clamped.device_meta()
    assert meta["eval_start"] == -0.5 and meta["inv_resolution"] == 2.0
    # zero outside the sampled window when not wrapping
    assert clamped.evaluate(np.array([-1.0, 10.0]))[:, 0].tolist() == [0.0, 0.0]
    periodic = ArrayInterpolator(np.float64, {"time": np.arange(6) * 0.5, "F": np.array([0, 1, 2, 1, 0, 0.0])},
                                 ["F"])
    assert periodic.boundary_condition == "periodic" and periodic.num_segments == 5


@pytest.mark.parametrize("d,msg", [
    ({"F": np.zeros(5)}, "time array or driver_sample_period"),
    ({"F": np.zeros(5), "time": np.arange(5.0), "driver_sample_period": 1.0}, "Only one of"),
    ({"F": np.zeros(5), "time": np.array([0.0, 1.0, 0.5, 2.0, 3.0])}, "strictly increasing"),
    ({"F": np.zeros(5), "time": np.array([0.0, 1.0, 2.5, 3.0, 4.0])}, "uniformly spaced"),
    ({"F": np.zeros((5, 2)), "driver_sample_period": 1.0}, "one-dimensional"),
    ({"F": np.zeros(3), "driver_sample_period": 1.0, "order": 3}, r"order \+ 1 samples"),
    ({"F": np.array([0.0, 1.0, 2.0, 3.0, 4.0]), "driver_sample_period": 1.0, "wrap": True}, "first and last"),
    ({"F": np.zeros(5), "driver_sample_period": 1.0, "wrap": False, "boundary_condition": "periodic"},
     "require wrap=True"),
    ({"G": np.zeros(5), "driver_sample_period": 1.0}, "not drivers of the system"),
])
def test_validation(d, msg):
    with pytest.raises(ValueError, match=msg):
        ArrayInterpolator(np.float64, d, ["F"])
