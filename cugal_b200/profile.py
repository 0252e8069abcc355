"""Phase timing and Sinkhorn statistics (reference ``cugal/profile.py:14-97``).

Same classes and fields as the reference.  The difference is when the device is
synchronised: the reference calls ``torch.cuda.synchronize()`` inside every
``log_time`` (``cugal/profile.py:45-48``), which serialises the host with the
GPU after every phase.  Here ``log_time`` only records a CUDA event pair on the
current stream; ``resolve()`` synchronises once and folds the pairs into
``phase_times``.  ``cugal()`` calls ``resolve()`` before it returns, so callers
see the same populated object.  Plotting and CSV helpers of the reference
(``cugal/profile.py:100-172``) are presentation code and are not mirrored.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from enum import Enum
from time import time

import torch


class Phase(Enum):
    FEATURE_EXTRACTION = "FEATURE_EXTRACTION"
    SINKHORN = "SINKHORN"
    HUNGARIAN = "HUNGARIAN"
    GRADIENT = "GRADIENT"


@dataclass
class SinkhornProfile:
    errors: list[float] = field(default_factory=list)
    iteration_count: int = 0
    time: float = 0.0
    # column-marginal L1 error of the returned plan, measured in FP32 (after the
    # polish sweeps when the solve streamed a reduced-precision cost)
    final_error: float = float("nan")

    @staticmethod
    def average(profiles: list["SinkhornProfile"]) -> "SinkhornProfile":
        t = sum(p.time for p in profiles) / len(profiles)
        count = int(sum(p.iteration_count for p in profiles) / len(profiles))
        return SinkhornProfile([], count, t)


class TimeStamp:
    """A point in time: a CUDA event on the current stream, or host time."""

    def __init__(self, device: str):
        if "cuda" in device:
            self.time = torch.cuda.Event(enable_timing=True)
            self.time.record()
        else:
            self.time = time()
        self.device = device

    def is_cuda_event(self) -> bool:
        return isinstance(self.time, torch.cuda.Event)

    def elapsed_seconds(self, earlier: "TimeStamp") -> float:
        if self.is_cuda_event():
            self.time.synchronize()
            return earlier.time.elapsed_time(self.time) / 1000
        return self.time - earlier.time


@dataclass
class Profile:
    sinkhorn_profiles: list[SinkhornProfile] = field(default_factory=list)
    phase_times: dict[Phase, float] = field(default_factory=dict)
    time: float = 0.0
    max_memory: int | None = None
    frank_wolfe_iterations: int = 0
    sparsity: float = 0.0
    # Event pairs not yet folded into phase_times (not part of to_dict()).
    _pending: list = field(default_factory=list, repr=False, compare=False)
    # Frank-Wolfe step of every update, 2/(2+it) or the line-search minimiser
    # (not part of to_dict(): the reference's Profile has no such field).
    _steps: list = field(default_factory=list, repr=False, compare=False)

    @property
    def frank_wolfe_steps(self) -> list[float]:
        return list(self._steps)

    def log_time(self, start_time: TimeStamp, phase: Phase):
        now = TimeStamp(start_time.device)
        if now.is_cuda_event():
            self._pending.append((phase, start_time, now))
        else:
            self.phase_times[phase] = self.phase_times.get(phase, 0.0) + now.elapsed_seconds(start_time)

    def resolve(self):
        """Synchronise once and fold all recorded event pairs into phase_times."""
        if self._pending:
            self._pending[-1][2].time.synchronize()
            for phase, start, end in self._pending:
                self.phase_times[phase] = self.phase_times.get(phase, 0.0) + \
                    start.time.elapsed_time(end.time) / 1000
            self._pending.clear()

    def to_dict(self) -> dict:
        self.resolve()
        d = {f.name: getattr(self, f.name) for f in dataclasses.fields(self) if not f.name.startswith("_")}
        # the reference's SinkhornProfile fields only (its from_dict takes no others),
        # so result files written here load there
        d["sinkhorn_profiles"] = [{"errors": list(p.errors), "iteration_count": p.iteration_count, "time": p.time}
                                  for p in self.sinkhorn_profiles]
        d["phase_times"] = {phase.value: t for phase, t in self.phase_times.items()}
        return d

    @classmethod
    def from_dict(cls, d: dict):
        d = dict(d)
        known = {f.name for f in dataclasses.fields(SinkhornProfile)}
        d["sinkhorn_profiles"] = [SinkhornProfile(**{k: v for k, v in p.items() if k in known})
                                  for p in d["sinkhorn_profiles"]]
        d["phase_times"] = {Phase[p]: t for p, t in d["phase_times"].items()}
        return cls(**d)

    @staticmethod
    def average(profiles: list["Profile"]) -> "Profile":
        for p in profiles:
            p.resolve()
        phase_times = {ph: sum(p.phase_times[ph] for p in profiles) / len(profiles)
                       for ph in profiles[0].phase_times}
        t = sum(p.time for p in profiles) / len(profiles)
        max_memory = max((p.max_memory for p in profiles if p.max_memory is not None), default=0)
        count = len(profiles[0].sinkhorn_profiles)
        fw = sum(p.frank_wolfe_iterations for p in profiles) / len(profiles)
        sparsity = sum(p.sparsity for p in profiles) / len(profiles)
        if all(len(p.sinkhorn_profiles) == count for p in profiles):
            sinkhorn = [SinkhornProfile.average([p.sinkhorn_profiles[i] for p in profiles]) for i in range(count)]
        else:
            sinkhorn = []
        return Profile(sinkhorn, phase_times, t, max_memory, fw, sparsity)
