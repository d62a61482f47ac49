"""Host-side result container (``batchsolving/solveresult.py:194-820``).

Arrays keep the reference's stride order ``[time, variable, run]`` for
time-domain outputs and ``[summary, variable * metric, run]`` for
summaries.  Runs whose status word is non-zero are NaN-masked unless
``nan_error_trajectories=False`` (``solveresult.py:373-404``); the time
column is left readable.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .result_codes import decode_status_codes


@dataclass
class SolveSpec:
    """Settings a solve ran with."""

    algorithm: str
    duration: float
    warmup: float
    t0: float
    dt: Optional[float]
    dt_min: float
    dt_max: float
    save_every: Optional[float]
    summarise_every: Optional[float]
    sample_summaries_every: Optional[float]
    atol: np.ndarray
    rtol: np.ndarray
    output_types: List[str]
    saved_states: List[str]
    saved_observables: List[str]
    summarised_states: List[str]
    summarised_observables: List[str]
    precision: type
    mixed_precision: bool = False
    kernel: str = "persistent"


@dataclass
class SolveResult:
    state: Optional[np.ndarray] = None              # includes a trailing time column when saved
    observables: Optional[np.ndarray] = None
    state_summaries: Optional[np.ndarray] = None
    observable_summaries: Optional[np.ndarray] = None
    iteration_counters: Optional[np.ndarray] = None
    status_codes: Optional[np.ndarray] = None
    time_domain_legend: Dict[int, str] = field(default_factory=dict)
    summaries_legend: Dict[int, str] = field(default_factory=dict)
    solve_settings: Optional[SolveSpec] = None
    save_time: bool = False
    totals: Optional[Dict[str, int]] = None
    kernel_ms: Optional[float] = None

    def mask_error_runs(self) -> None:
        codes = self.status_codes
        if codes is None or codes.size == 0:
            return
        bad = np.where(codes != 0)[0]
        if bad.size == 0:
            return
        for arr in (self._state_less_time, self.observables, self.state_summaries, self.observable_summaries):
            if arr is not None and arr.size:
                arr[:, :, bad] = np.nan

    @property
    def _state_less_time(self) -> Optional[np.ndarray]:
        if self.state is None:
            return None
        return self.state[:, :-1, :] if self.save_time else self.state

    @property
    def time(self) -> Optional[np.ndarray]:
        if not self.save_time or self.state is None:
            return None
        return self.state[:, -1, :]

    @staticmethod
    def _combine(*arrays) -> np.ndarray:
        active = [a for a in arrays if a is not None and a.size > 0]
        if not active:
            return np.array([])
        if len(active) == 1:
            return active[0]
        return np.concatenate(active, axis=1)

    @property
    def time_domain_array(self) -> np.ndarray:
        return self._combine(self._state_less_time, self.observables)

    @property
    def summaries_array(self) -> np.ndarray:
        return self._combine(self.state_summaries, self.observable_summaries)

    @property
    def status_messages(self) -> Dict[int, List[str]]:
        return decode_status_codes(self.status_codes)

    def as_numpy(self) -> Dict[str, Optional[np.ndarray]]:
        return {
            "time_domain_array": self.time_domain_array,
            "summaries_array": self.summaries_array,
            "time": self.time,
            "iteration_counters": self.iteration_counters,
            "status_codes": self.status_codes,
            "time_domain_legend": dict(self.time_domain_legend),
            "summaries_legend": dict(self.summaries_legend),
        }

    def as_pandas(self) -> Dict[str, "object"]:
        import pandas as pd
        out = {}
        td = self.time_domain_array
        if td.size:
            frames = []
            for r in range(td.shape[2]):
                df = pd.DataFrame(td[:, :, r], columns=[self.time_domain_legend.get(i, str(i)) for i in range(td.shape[1])])
                df["run"] = r
                if self.time is not None:
                    df["time"] = self.time[:, r]
                frames.append(df)
            out["time_domain"] = pd.concat(frames, ignore_index=True)
        sm = self.summaries_array
        if sm.size:
            frames = []
            for r in range(sm.shape[2]):
                df = pd.DataFrame(sm[:, :, r], columns=[self.summaries_legend.get(i, str(i)) for i in range(sm.shape[1])])
                df["run"] = r
                frames.append(df)
            out["summaries"] = pd.concat(frames, ignore_index=True)
        return out


def merge_results(parts) -> SolveResult:
    """Reassemble one family's SolveResult from sub-results over disjoint run
    index sets ``[(result, run_indices), ...]`` (arrays promoted to the
    widest dtype among the parts; totals summed)."""
    import copy
    first = parts[0][0]
    n = sum(len(idx) for _, idx in parts)
    res = copy.copy(first)
    for name in ("state", "observables", "state_summaries", "observable_summaries", "iteration_counters"):
        arrs = [getattr(r, name) for r, _ in parts]
        if any(a is None for a in arrs):
            setattr(res, name, None)
            continue
        dtype = np.result_type(*arrs)
        full = np.empty(arrs[0].shape[:-1] + (n,), dtype=dtype)
        for a, (_, idx) in zip(arrs, parts):
            full[..., idx] = a
        setattr(res, name, full)
    status = np.empty(n, dtype=first.status_codes.dtype)
    for r, idx in parts:
        status[idx] = r.status_codes
    res.status_codes = status
    if all(r.totals is not None for r, _ in parts):
        res.totals = {k: sum(r.totals[k] for r, _ in parts) for k in first.totals}
    return res
