"""Array drivers: piecewise-polynomial interpolation of sampled inputs.

Host side of the reference's ``ArrayInterpolator``
(src/cubie/array_interpolator.py:151-1134).  A driver dictionary holds one
1-D sample array per driver symbol of the system, plus either ``"time"``
(uniformly spaced sample times) or ``"driver_sample_period"`` and ``"t0"``,
and optionally ``"order"`` (default 3), ``"wrap"`` (default True) and
``"boundary_condition"`` ("natural", "periodic", "clamped", "not-a-knot";
default "periodic" when wrapping, "clamped" otherwise; :281-307).

Coefficients: one polynomial of degree ``order`` per segment between
consecutive samples, in the local variable tau in [0, 1), fitted jointly:
values at both ends of every segment, continuity of derivatives 1..order-1
at interior knots, and ``order - 1`` end conditions (:899-1087).  Clamped,
non-wrapping inputs are padded with a zero sample at both ends (two ghost
segments) so the signal ramps to zero outside the sampled window.  The
system is assembled with one block of rows per segment and solved as a
sparse system in FP64 (the reference assembles the same equations and
solves them densely in the working precision); the result is stored
segment-major, ``[segment, driver, power]``, in the working precision.

Device evaluation (``Drivers<Cfg>`` in csrc/device/cbx_steps.cuh) follows
``evaluate_all`` / ``evaluate_time_derivative`` (:463-550): scaled time
(t - eval_start) / period, segment = floor (modulo the segment count when
wrapping, clamped otherwise), Horner in tau, zero outside the window when
not wrapping.
"""

from __future__ import annotations

import math
from typing import Any, Dict, Optional, Sequence

import numpy as np

BOUNDARY_CONDITIONS = ("natural", "periodic", "clamped", "not-a-knot")
CONFIG_KEYS = ("order", "wrap", "boundary_condition")
TIME_KEYS = ("time", "driver_sample_period", "t0")


def _falling(order: int) -> np.ndarray:
    """falling[p, d] = p (p - 1) ... (p - d + 1): d-th derivative of tau^p at 1."""
    f = np.zeros((order + 1, order + 1))
    f[:, 0] = 1.0
    for d in range(1, order + 1):
        for p in range(d, order + 1):
            f[p, d] = f[p, d - 1] * (p - (d - 1))
    return f


def spline_coefficients(samples: np.ndarray, order: int, boundary_condition: str) -> np.ndarray:
    """Coefficients ``[segment, input, power]`` through ``samples``
    ``[n_samples, n_inputs]`` (float64 solve)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve

    y = np.asarray(samples, dtype=np.float64)
    nseg = y.shape[0] - 1
    nin = y.shape[1]
    K = order + 1
    nc = nseg * K
    fall = _falling(order)
    rows, cols, vals = [], [], []
    rhs = np.zeros((nc, nin))
    r = 0

    def put(row, col, v):
        rows.append(row)
        cols.append(col)
        vals.append(v)

    for s in range(nseg):
        # value at the left and right end of segment s
        put(r, s * K, 1.0)
        rhs[r] = y[s]
        r += 1
        for p in range(K):
            put(r, s * K + p, 1.0)
        rhs[r] = y[s + 1]
        r += 1
        # continuity of derivatives 1..order-1 into segment s + 1
        if s < nseg - 1:
            for d in range(1, order):
                for p in range(d, K):
                    put(r, s * K + p, fall[p, d])
                put(r, (s + 1) * K + d, -fall[d, d])
                r += 1
    if boundary_condition in ("natural", "clamped"):
        remaining = order - 1
        d = 2 if boundary_condition == "natural" else 1
        while remaining > 0 and d <= order:
            put(r, d, fall[d, d])                      # derivative d at the start
            r += 1
            remaining -= 1
            if remaining == 0:
                break
            base = (nseg - 1) * K
            for p in range(d, K):                      # derivative d at the end
                put(r, base + p, fall[p, d])
            r += 1
            remaining -= 1
            d += 1
    elif boundary_condition == "periodic":
        base = (nseg - 1) * K
        for d in range(1, order):
            for p in range(d, K):
                put(r, base + p, fall[p, d])
            put(r, d, -fall[d, d])
            r += 1
    elif boundary_condition == "not-a-knot":
        needed = order - 1
        added = 0
        for q in range(1, order):
            if added >= needed:
                break
            # q-th forward difference of the leading coefficients vanishes
            for off in range(q + 1):
                put(r, off * K + order, float((-1) ** (q - off) * math.comb(q, off)))
            r += 1
            added += 1
            if added >= needed:
                break
            for off in range(q + 1):
                seg = nseg - 1 - (q - off)
                put(r, seg * K + order, float((-1) ** (q - off) * math.comb(q, off)))
            r += 1
            added += 1
    else:
        raise ValueError(f"boundary_condition must be one of {BOUNDARY_CONDITIONS}")
    if r != nc:
        raise ValueError("the spline system is not square: check the boundary condition and sample count")
    A = csr_matrix((vals, (rows, cols)), shape=(nc, nc))
    sol = spsolve(A.tocsc(), rhs)
    sol = np.asarray(sol).reshape(nc, nin)
    return np.ascontiguousarray(sol.reshape(nseg, K, nin).transpose(0, 2, 1))


class ArrayInterpolator:
    """Interpolated drivers for one system (reference ``ArrayInterpolator``)."""

    def __init__(self, precision, input_dict: Dict[str, Any], driver_names: Sequence[str]):
        self.precision = np.dtype(precision).type
        p = self.precision
        self.order = int(input_dict.get("order", 3))
        if self.order < 0:
            raise ValueError("order must be >= 0")
        self.wrap = bool(input_dict.get("wrap", True))
        bc = input_dict.get("boundary_condition")
        if bc is None:
            bc = "periodic" if self.wrap else "clamped"
        if bc not in BOUNDARY_CONDITIONS:
            raise ValueError(f"boundary_condition must be one of {BOUNDARY_CONDITIONS}")
        self.boundary_condition = bc
        names = list(driver_names)
        unknown = [k for k in input_dict if k not in CONFIG_KEYS and k not in TIME_KEYS and k not in names]
        if unknown:
            raise ValueError(f"driver arrays {unknown} are not drivers of the system {names}")
        missing = [nm for nm in names if nm not in input_dict]
        if missing:
            raise ValueError(f"no samples given for drivers {missing}")
        arrays = []
        for nm in names:
            a = np.asarray(input_dict[nm], dtype=p)
            if a.ndim != 1:
                raise ValueError(f"Forcing array {nm} must be one-dimensional.")
            arrays.append(a)
        if any(a.shape[0] != arrays[0].shape[0] for a in arrays):
            raise ValueError("All forcing vectors must have the same length / be sampled on the same grid")
        self.input_array = np.column_stack(arrays) if arrays else np.zeros((0, 0), p)
        if self.input_array.shape[0] < self.order + 1:
            raise ValueError("At least order + 1 samples are required to construct splines.")
        self.driver_sample_period, self.t0 = self._time(input_dict)
        pad = (not self.wrap) and bc == "clamped"
        if bc == "periodic":
            if not self.wrap:
                raise ValueError("Periodic boundary conditions require wrap=True so that the input repeats "
                                 "after the final segment.")
            if not np.allclose(self.input_array[0], self.input_array[-1]):
                raise ValueError("Periodic boundary conditions require the first and last samples to match.")
        samples = self.input_array
        if pad:
            z = np.zeros((1, samples.shape[1]), p)
            samples = np.vstack((z, samples, z))
        self.num_segments = samples.shape[0] - 1
        self.coefficients = spline_coefficients(samples, self.order, bc).astype(p)

    def _time(self, d: Dict[str, Any]):
        if "driver_sample_period" in d and "time" in d:
            raise ValueError("Only one of driver_sample_period or time should be provided.")
        if "driver_sample_period" in d:
            return float(d["driver_sample_period"]), float(d.get("t0", 0.0))
        if "time" in d:
            t = np.asarray(d["time"], dtype=np.float64)
            if t.ndim != 1:
                raise ValueError("Time array must be one-dimensional.")
            if t.shape[0] != self.input_array.shape[0]:
                raise ValueError("Time array length must match the number of samples in provided input vectors.")
            dt = np.diff(t)
            if np.any(dt <= 0.0):
                raise ValueError("Time array must be strictly increasing.")
            if not np.allclose(dt, np.full_like(dt, dt[0]), rtol=1e-6, atol=1e-6):
                raise ValueError("Time array must be uniformly spaced.")
            return float(dt[0]), float(t[0])
        raise ValueError("Either a time array or driver_sample_period must be provided.")

    @classmethod
    def from_system(cls, system, drivers: Optional[Dict[str, Any]], precision) -> "ArrayInterpolator":
        if drivers is None:
            raise ValueError(f"the system has drivers {system.driver_names}: pass their samples in ``drivers``")
        if isinstance(drivers, ArrayInterpolator):
            return drivers
        return cls(precision, dict(drivers), system.driver_names)

    @property
    def num_inputs(self) -> int:
        return self.input_array.shape[1]

    def device_meta(self) -> Dict[str, Any]:
        """Compile-time constants of the device evaluator (:437-451)."""
        p = self.precision
        res = p(self.driver_sample_period)
        inv = p(p(1.0) / res)
        pad = (not self.wrap) and self.boundary_condition == "clamped"
        start = p(p(self.t0) - (res if pad else p(0.0)))
        return dict(order=self.order, num_segments=self.num_segments, eval_start=float(start),
                    inv_resolution=float(inv), wrap=self.wrap)

    def evaluate(self, times, derivative: bool = False) -> np.ndarray:
        """Host evaluation ``[len(times), n_inputs]`` in the working precision,
        the same arithmetic as the device evaluator."""
        p = self.precision
        m = self.device_meta()
        t = np.asarray(times, dtype=p)
        scaled = (t - p(m["eval_start"])) * p(m["inv_resolution"])
        fl = np.floor(scaled)
        idx = fl.astype(np.int64)
        n = self.num_segments
        if self.wrap:
            seg = np.mod(idx, n)
            tau = (scaled - fl).astype(p)
            in_range = np.ones(t.shape, bool)
        else:
            in_range = (scaled >= 0) & (scaled <= n)
            seg = np.clip(idx, 0, n - 1)
            tau = (scaled - seg.astype(p)).astype(p)
        c = self.coefficients[seg]            # [times, inputs, power]
        acc = np.zeros((t.shape[0], self.num_inputs), p)
        if derivative:
            for k in range(self.order, 0, -1):
                acc = acc * tau[:, None] + p(k) * c[:, :, k]
            acc = acc * p(m["inv_resolution"])
        else:
            for k in range(self.order, -1, -1):
                acc = acc * tau[:, None] + c[:, :, k]
        return np.where(in_range[:, None], acc, p(0))
