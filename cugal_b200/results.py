"""Result files in the reference's format (``benchmark/experiment.py:20-31,145-162,
404-430,513-555``), so alignments run here can be compared with, and stored
beside, the reference's ``benchmark/results/*.json``.

A file is ``{"experiment": ..., "commit": ..., "time": ..., "results": ...}``:
the experiment (algorithms with their ``Config``, graphs as ``{"kind",
"parameters"}``, noise levels and run options) and, for each graph, noise level
and algorithm, one ``Result`` (ICS, EC, S3, accuracy, ``Profile``).  The graph
generators and the dataset loaders of the reference's harness are not part of
this package; the experiment's graphs and noise levels are carried as the plain
dictionaries the reference writes.
"""

from __future__ import annotations

import dataclasses
import datetime
import json
import subprocess
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable

from .config import Config
from .metrics import Result


@dataclass(frozen=True)
class NoiseLevel:
    """``benchmark/experiment.py:20-31``."""
    source_noise: float
    target_noise: float
    refill_edges: bool

    def to_dict(self) -> dict:
        return dataclasses.asdict(self)


ADDITIONS_KEY = "config_b200"


@dataclass(frozen=True)
class Algorithm:
    """``benchmark/experiment.py:145-162``: a ``Config`` and whether FUGAL's own
    (CPU) implementation ran instead of cuGAL's.  ``"config"`` holds the
    reference's fields only (its loader rejects others); the fields added here
    go under ``"config_b200"``, which the reference's loader ignores."""
    config: Config
    use_fugal: bool = False

    def to_dict(self) -> dict:
        ref, added = self.config.split_dict()
        return {"use_fugal": self.use_fugal, "config": ref, ADDITIONS_KEY: added}

    @classmethod
    def from_dict(cls, d: dict) -> "Algorithm":
        merged = {**d["config"], **d.get(ADDITIONS_KEY, {})}
        return cls(config=Config.from_dict(merged), use_fugal=d["use_fugal"])


@dataclass
class Experiment:
    """``benchmark/experiment.py:404-430`` without the runner: graphs stay the
    reference's ``{"kind": ..., "parameters": {...}}`` dictionaries."""
    algorithms: list[Algorithm]
    graphs: list[dict]
    noise_levels: list[NoiseLevel]
    debug: bool = False
    seed: int | None = None
    save_alignment: bool = False
    num_runs: int = 1

    def to_dict(self) -> dict:
        return {"algorithms": [a.to_dict() for a in self.algorithms],
                "graphs": [dict(g) for g in self.graphs],
                "noise_levels": [n.to_dict() for n in self.noise_levels],
                "debug": self.debug, "seed": self.seed, "save_alignment": self.save_alignment,
                "num_runs": self.num_runs}

    @classmethod
    def from_dict(cls, d: dict) -> "Experiment":
        d = dict(d)
        d["algorithms"] = [Algorithm.from_dict(a) for a in d["algorithms"]]
        d["graphs"] = [dict(g) for g in d["graphs"]]
        d["noise_levels"] = [NoiseLevel(**n) for n in d["noise_levels"]]
        return cls(**d)


def last_commit() -> str:
    """``git rev-parse HEAD`` of the working directory, or "" (``experiment.py:395-400``)."""
    try:
        out = subprocess.run(["git", "rev-parse", "HEAD"], capture_output=True, text=True, check=True)
        return out.stdout.strip()
    except (subprocess.CalledProcessError, OSError):
        return ""


@dataclass
class ExperimentResults:
    """``benchmark/experiment.py:513-555``; ``results[graph][noise level][algorithm]``."""
    experiment: Experiment
    commit: str = ""
    time: str = field(default_factory=lambda: str(datetime.datetime.now()))
    results: list[list[list[Result]]] = field(default_factory=list)

    def all_results(self) -> Iterable[tuple[dict, NoiseLevel, Algorithm, Result]]:
        for graph, per_graph in zip(self.experiment.graphs, self.results):
            for level, per_level in zip(self.experiment.noise_levels, per_graph):
                for algorithm, result in zip(self.experiment.algorithms, per_level):
                    yield graph, level, algorithm, result

    def name(self) -> str:
        return "-".join(g["kind"] for g in self.experiment.graphs) + "-" + self.time.replace(" ", "-")

    def to_dict(self) -> dict:
        return {"experiment": self.experiment.to_dict(), "commit": self.commit, "time": self.time,
                "results": [[[r.to_dict() for r in c] for c in b] for b in self.results]}

    @classmethod
    def from_dict(cls, d: dict) -> "ExperimentResults":
        return cls(experiment=Experiment.from_dict(d["experiment"]), commit=d["commit"], time=d["time"],
                   results=[[[Result.from_dict(r) for r in c] for c in b] for b in d["results"]])

    def dump(self, folder: str | Path) -> Path:
        path = Path(folder) / (self.name() + ".json")
        path.write_text(json.dumps(self.to_dict(), indent=4))
        return path

    @classmethod
    def load(cls, path: str | Path) -> "ExperimentResults":
        return cls.from_dict(json.loads(Path(path).read_text()))
