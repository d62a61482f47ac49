"""Output types, summary metrics and the save/summary schedule.

* Output-type parsing mirrors ``outputhandling/output_config.py:120-151``:
  ``state``, ``observables``, ``time`` and ``iteration_counters`` are direct
  outputs; any name starting with a registered metric is a summary metric,
  with an optional ``[n]`` parameter (``peaks[3]``).
* Summary metrics follow ``outputhandling/summarymetrics/*.py``: each has a
  per-variable accumulation buffer, an output width, an update rule applied
  at every summary sample and a save rule applied every
  ``samples_per_summary`` samples.  Combined metrics replace requested
  subsets (``mean``+``std`` -> ``mean_std`` ...) as in ``metrics.py:345-467``.
* Event counts and stop times follow ``SingleIntegratorRun.py:153-292``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple
import warnings

import numpy as np

DIRECT_TYPES = ("state", "observables", "time", "iteration_counters")


@dataclass(frozen=True)
class Metric:
    name: str
    buf: object          # int or callable(param) -> int
    out: object
    update: str          # C++ statements; v: value, b: buffer, idx: sample index, P: param
    save: str            # C++ statements; b: buffer, o: outputs, n: samples per summary, P: param
    legend: Tuple[str, ...] = ()

    def buffer_size(self, param: int) -> int:
        return self.buf(param) if callable(self.buf) else int(self.buf)

    def output_size(self, param: int) -> int:
        return self.out(param) if callable(self.out) else int(self.out)


_SHIFTED_UPDATE = """if (idx == 0) { b[0] = v; b[1] = R(0); b[2] = R(0); }
{ const R sv = v - b[0]; b[1] += sv; b[2] += sv * sv; }"""

METRICS: Dict[str, Metric] = {
    "mean": Metric("mean", 1, 1, "b[0] += v;",
                   "o[0] = R(double(b[0]) / double(n)); b[0] = R(0);", ("mean",)),
    "max": Metric("max", 1, 1, "if (v > b[0]) b[0] = v;",
                  "o[0] = b[0]; b[0] = R(-1.0e30);", ("max",)),
    "min": Metric("min", 1, 1, "if (v < b[0]) b[0] = v;",
                  "o[0] = b[0]; b[0] = R(1.0e30);", ("min",)),
    "rms": Metric("rms", 1, 1,
                  "{ R s = b[0]; if (idx == 0) s = R(0); s += v * v; b[0] = s; }",
                  "o[0] = R(sqrt(double(b[0]) / double(n))); b[0] = R(0);", ("rms",)),
    "std": Metric("std", 3, 1, _SHIFTED_UPDATE,
                  """{ const R ms = R(double(b[1]) / double(n)); const R mss = R(double(b[2]) / double(n));
const R var = mss - ms * ms; o[0] = R(sqrt(double(var))); b[0] = b[0] + ms; b[1] = R(0); b[2] = R(0); }""",
                  ("std",)),
    "mean_std": Metric("mean_std", 3, 2, _SHIFTED_UPDATE,
                       """{ const R sh = b[0]; const R ms = R(double(b[1]) / double(n)); const R mss = R(double(b[2]) / double(n));
const R mean = sh + ms; const R var = mss - ms * ms; o[0] = mean; o[1] = R(sqrt(double(var)));
b[0] = mean; b[1] = R(0); b[2] = R(0); }""", ("mean", "std")),
    "mean_std_rms": Metric("mean_std_rms", 3, 3, _SHIFTED_UPDATE,
                           """{ const R sh = b[0]; const R ms = R(double(b[1]) / double(n)); const R mss = R(double(b[2]) / double(n));
const R mean = sh + ms; const R var = mss - ms * ms; const R msq = mss + R(2) * sh * ms + sh * sh;
o[0] = mean; o[1] = R(sqrt(double(var))); o[2] = R(sqrt(double(msq))); b[0] = mean; b[1] = R(0); b[2] = R(0); }""",
                           ("mean", "std", "rms")),
    "std_rms": Metric("std_rms", 3, 2, _SHIFTED_UPDATE,
                      """{ const R sh = b[0]; const R ms = R(double(b[1]) / double(n)); const R mss = R(double(b[2]) / double(n));
const R var = mss - ms * ms; const R msq = mss + R(2) * sh * ms + sh * sh;
o[0] = R(sqrt(double(var))); o[1] = R(sqrt(double(msq))); b[0] = sh + ms; b[1] = R(0); b[2] = R(0); }""",
                      ("std", "rms")),
    "extrema": Metric("extrema", 2, 2, "if (v > b[0]) b[0] = v; if (v < b[1]) b[1] = v;",
                      "o[0] = b[0]; o[1] = b[1]; b[0] = R(-1.0e30); b[1] = R(1.0e30);", ("max", "min")),
    "max_magnitude": Metric("max_magnitude", 1, 1, "{ const R av = fabs(v); if (av > b[0]) b[0] = av; }",
                            "o[0] = b[0]; b[0] = R(0);", ("max_magnitude",)),
    "peaks": Metric(
        "peaks", lambda n: 3 + n, lambda n: n,
        """{ const R prev = b[0]; const R prev_prev = b[1]; const int pc = int(b[2]);
if (idx >= 2 && pc < P && prev_prev != R(0)) { if (prev > v && prev_prev < prev) {
#pragma unroll
  for (int q = 0; q < P; ++q) if (q == pc) b[3 + q] = R(idx - 1);
  b[2] = R(int(b[2]) + 1); } }
b[0] = v; b[1] = prev; }""",
        """
#pragma unroll
for (int q = 0; q < P; ++q) { o[q] = b[3 + q]; b[3 + q] = R(0); }
b[2] = R(0);""", ("peaks",)),
    "negative_peaks": Metric(
        "negative_peaks", lambda n: 3 + n, lambda n: n,
        """{ const R prev = b[0]; const R prev_prev = b[1]; const int pc = int(b[2]);
if (idx >= 2 && pc < P && prev_prev != R(0)) { if (prev < v && prev_prev > prev) {
#pragma unroll
  for (int q = 0; q < P; ++q) if (q == pc) b[3 + q] = R(idx - 1);
  b[2] = R(int(b[2]) + 1); } }
b[0] = v; b[1] = prev; }""",
        """
#pragma unroll
for (int q = 0; q < P; ++q) { o[q] = b[3 + q]; b[3 + q] = R(0); }
b[2] = R(0);""", ("negative_peaks",)),
}

# Finite-difference derivative metrics (dxdt_*.py, d2xdt2_*.py): the buffer
# keeps the previous sample(s) across summary windows; differences are
# unscaled until the save divides by the sample interval (squared for the
# second difference).  ``idx`` (the run's summary-sample counter) gates the
# first one or two samples, which have no history.
_D1 = "const R d = v - b[0];"
_D2 = "const R d = v - R(2.0) * b[0] + b[1];"
METRICS.update({
    "dxdt_max": Metric("dxdt_max", 2, 1, "{ " + _D1 + " if (d > b[1] && idx >= 1) b[1] = d; b[0] = v; }",
                       "o[0] = b[1] / R(DT_SAMPLE); b[1] = R(-1.0e30);", ("dxdt_max",)),
    "dxdt_min": Metric("dxdt_min", 2, 1, "{ " + _D1 + " if (d < b[1] && idx >= 1) b[1] = d; b[0] = v; }",
                       "o[0] = b[1] / R(DT_SAMPLE); b[1] = R(1.0e30);", ("dxdt_min",)),
    "dxdt_extrema": Metric(
        "dxdt_extrema", 3, 2,
        "{ " + _D1 + " if (d > b[1] && idx >= 1) b[1] = d; if (d < b[2] && idx >= 1) b[2] = d; b[0] = v; }",
        "o[0] = b[1] / R(DT_SAMPLE); o[1] = b[2] / R(DT_SAMPLE); b[1] = R(-1.0e30); b[2] = R(1.0e30);",
        ("dxdt_max", "dxdt_min")),
    "d2xdt2_max": Metric(
        "d2xdt2_max", 3, 1, "{ " + _D2 + " if (d > b[2] && idx >= 2) b[2] = d; b[1] = b[0]; b[0] = v; }",
        "{ const R s2 = R(DT_SAMPLE) * R(DT_SAMPLE); o[0] = b[2] / s2; b[2] = R(-1.0e30); }", ("d2xdt2_max",)),
    "d2xdt2_min": Metric(
        "d2xdt2_min", 3, 1, "{ " + _D2 + " if (d < b[2] && idx >= 2) b[2] = d; b[1] = b[0]; b[0] = v; }",
        "{ const R s2 = R(DT_SAMPLE) * R(DT_SAMPLE); o[0] = b[2] / s2; b[2] = R(1.0e30); }", ("d2xdt2_min",)),
    "d2xdt2_extrema": Metric(
        "d2xdt2_extrema", 4, 2,
        "{ " + _D2 + " if (d > b[2] && idx >= 2) b[2] = d; if (d < b[3] && idx >= 2) b[3] = d; "
        "b[1] = b[0]; b[0] = v; }",
        "{ const R s2 = R(DT_SAMPLE) * R(DT_SAMPLE); o[0] = b[2] / s2; o[1] = b[3] / s2; "
        "b[2] = R(-1.0e30); b[3] = R(1.0e30); }", ("d2xdt2_max", "d2xdt2_min")),
})

COMBINED = [
    (frozenset(["mean", "std", "rms"]), "mean_std_rms"),
    (frozenset(["mean", "std"]), "mean_std"),
    (frozenset(["std", "rms"]), "std_rms"),
    (frozenset(["max", "min"]), "extrema"),
    (frozenset(["dxdt_max", "dxdt_min"]), "dxdt_extrema"),
    (frozenset(["d2xdt2_max", "d2xdt2_min"]), "d2xdt2_extrema"),
]


def parse_output_types(output_types: Sequence[str]) -> Tuple[Dict[str, bool], Tuple[str, ...]]:
    """Split output types into direct-output flags and summary requests."""
    if isinstance(output_types, str):
        output_types = (output_types,)
    flags = {name: name in output_types for name in DIRECT_TYPES}
    summaries = []
    for ot in output_types:
        if any(ot.startswith(m) for m in METRICS):
            summaries.append(ot)
        elif ot not in DIRECT_TYPES:
            warnings.warn(f"Summary type '{ot}' is not implemented. Ignoring.")
    return flags, tuple(summaries)


@dataclass
class SummaryPlan:
    """Processed summary metrics with parameters and layout."""

    metrics: List[Tuple[Metric, int]] = field(default_factory=list)

    @staticmethod
    def empty() -> "SummaryPlan":
        return SummaryPlan([])

    @staticmethod
    def from_request(request: Sequence[str]) -> "SummaryPlan":
        clean: List[str] = []
        params: Dict[str, int] = {}
        for item in request:
            if "[" in item:
                name, rest = item.split("[", 1)
                try:
                    params[name] = int(rest.split("]")[0])
                except ValueError as exc:
                    raise ValueError(f"Parameter in '{item}' must be an integer.") from exc
                clean.append(name)
            else:
                clean.append(item)
                params.setdefault(item, 0)
        result: List[str] = []
        used = set()
        for m in clean:
            if m in used:
                continue
            done = False
            for members, combo in COMBINED:
                if m in members and members.issubset(clean) and combo not in result:
                    result.append(combo)
                    used |= members
                    params[combo] = 0
                    done = True
                    break
            if not done:
                result.append(m)
                used.add(m)
        metrics = []
        for name in result:
            if name not in METRICS:
                warnings.warn(f"Metric '{name}' is not registered. Skipping.")
                continue
            metrics.append((METRICS[name], params.get(name, 0)))
        return SummaryPlan(metrics)

    @property
    def buffer_per_var(self) -> int:
        return sum(m.buffer_size(p) for m, p in self.metrics)

    @property
    def output_per_var(self) -> int:
        return sum(m.output_size(p) for m, p in self.metrics)

    def legend(self) -> List[str]:
        out = []
        for m, p in self.metrics:
            if m.name in ("peaks", "negative_peaks"):
                out.extend(f"{m.name}[{i}]" for i in range(p))
            else:
                out.extend(m.legend)
        return out

    def device_struct(self, sample_every: float = 0.0) -> str:
        """The generated ``Summ`` struct; ``sample_every`` (the summary
        sample interval, already in the system precision) scales the
        derivative metrics."""
        lines = ["struct Summ {",
                 f"    static constexpr int BUF = {max(self.buffer_per_var, 1)};",
                 f"    static constexpr int OUT = {self.output_per_var};",
                 f"    static constexpr double DT_SAMPLE = {float(sample_every)!r};",
                 "    template <class R> static __device__ __forceinline__ void update(R v, R* buf, int idx) {",
                 "        (void)v; (void)buf; (void)idx;"]
        off = 0
        for m, p in self.metrics:
            lines.append(f"        {{ R* b = buf + {off}; const int P = {p}; (void)P;")
            lines.append("        " + m.update.replace("\n", "\n        "))
            lines.append("        }")
            off += m.buffer_size(p)
        lines.append("    }")
        lines.append("    template <class R> static __device__ __forceinline__ void save(R* buf, R* out, int n) {")
        lines.append("        (void)buf; (void)out; (void)n;")
        boff, ooff = 0, 0
        for m, p in self.metrics:
            lines.append(f"        {{ R* b = buf + {boff}; R* o = out + {ooff}; const int P = {p}; (void)P;")
            lines.append("        " + m.save.replace("\n", "\n        "))
            lines.append("        }")
            boff += m.buffer_size(p)
            ooff += m.output_size(p)
        lines.append("    }")
        lines.append("};")
        return "\n".join(lines)


# ---------------------------------------------------------------------------
# Schedule helpers (SingleIntegratorRun.py:153-292)
# ---------------------------------------------------------------------------
def regular_event_count(duration: float, interval: float, precision) -> int:
    """Events of ``interval`` in ``duration`` after casting both to the
    working precision, with a 4-eps allowance capped below one half."""
    precision = np.dtype(precision).type
    total = np.float64(precision(duration)) / np.float64(precision(interval))
    allowance = min(4.0 * float(np.finfo(precision).eps) * total, 0.49)
    return int(np.floor(total + allowance))


def output_length(duration: float, save_every: Optional[float], save_last: bool, precision) -> int:
    regular = regular_event_count(duration, save_every, precision) if save_every is not None else 0
    return regular + 1 + (1 if save_last else 0)


def save_stop_time(duration, settling_time, t0, save_every, precision) -> float:
    start = np.float64(settling_time) + np.float64(t0)
    if save_every is None:
        return float(start + np.float64(np.dtype(precision).type(duration)))
    events = regular_event_count(duration, save_every, precision)
    return float(start + (events + 0.5) * np.float64(np.dtype(precision).type(save_every)))


def summary_stop_time(duration, settling_time, t0, sample_every, precision) -> float:
    start = np.float64(settling_time) + np.float64(t0)
    if sample_every is None:
        return float(start + np.float64(np.dtype(precision).type(duration)))
    events = regular_event_count(duration, sample_every, precision)
    return float(start + (events + 0.5) * np.float64(np.dtype(precision).type(sample_every)))


def summaries_length(duration, sample_every, samples_per_summary, precision) -> int:
    if sample_every is None:
        return 0
    updates = regular_event_count(duration, sample_every, precision)
    return updates // max(samples_per_summary, 1)
