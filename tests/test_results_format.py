"""Result files in the reference's format (benchmark/experiment.py:513-555):
a sample of the reference's own results files (tests/golden/make_results_golden.py)
loads here and writes back unchanged, configurations keep exactly the reference's
fields under "config", and profiles carry only fields the reference's loader takes."""

import json
from pathlib import Path

import pytest

from cugal_b200.config import REFERENCE_FIELDS, Config, HungarianMethod, SinkhornMethod
from cugal_b200.metrics import Result
from cugal_b200.profile import Phase, Profile, SinkhornProfile
from cugal_b200.results import ADDITIONS_KEY, Algorithm, Experiment, ExperimentResults, NoiseLevel

SAMPLE = json.loads((Path(__file__).resolve().parent / "golden" / "reference_results_sample.json").read_text())


def _strip_additions(d):
    d = json.loads(json.dumps(d))
    for a in d["experiment"]["algorithms"]:
        a.pop(ADDITIONS_KEY, None)
    return d


@pytest.mark.parametrize("name", sorted(SAMPLE))
def test_reference_file_round_trip(name):
    original = SAMPLE[name]
    res = ExperimentResults.from_dict(json.loads(json.dumps(original)))
    back = _strip_additions(res.to_dict())
    for key in original["experiment"]:
        assert back["experiment"][key] == original["experiment"][key], key
    assert back["results"] == original["results"]
    assert (back["commit"], back["time"]) == (original["commit"], original["time"])
    for a in res.to_dict()["experiment"]["algorithms"]:
        assert tuple(a["config"]) == REFERENCE_FIELDS
        assert set(a[ADDITIONS_KEY]) == {"stream_dtype", "polish_sweeps", "fp32_warmup_sweeps", "reabsorb_every",
                                         "lap_candidates", "line_search"}
    assert [r.accuracy for _, _, _, r in res.all_results()] == \
        [r["accuracy"] for g in original["results"] for lv in g for r in lv]


def test_own_results_round_trip(tmp_path):
    import torch
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, use_sparse_adjacency=True,
                 hungarian_method=HungarianMethod.SCIPY, stream_dtype=torch.bfloat16, line_search=True)
    prof = Profile(sinkhorn_profiles=[SinkhornProfile([0.5, 0.01], 20, 0.1, final_error=3e-5)],
                   phase_times={Phase.SINKHORN: 1.5, Phase.GRADIENT: 0.5}, time=2.25, frank_wolfe_iterations=150,
                   sparsity=0.9)
    exp = Experiment(algorithms=[Algorithm(cfg)], graphs=[{"kind": "NEWMAN_WATTS", "parameters": {"n": 64}}],
                     noise_levels=[NoiseLevel(0.0, 0.05, True)], seed=7)
    res = ExperimentResults(exp, commit="abc", time="2026-01-01 00:00:00", results=[[[Result(0.9, 0.8, 0.7, 1.0, prof)]]])
    d = res.to_dict()
    # the reference's SinkhornProfile(**p) takes errors, iteration_count, time only
    assert set(d["results"][0][0][0]["profile"]["sinkhorn_profiles"][0]) == {"errors", "iteration_count", "time"}
    path = res.dump(tmp_path)
    assert path.name == "NEWMAN_WATTS-2026-01-01-00:00:00.json"
    back = ExperimentResults.load(path)
    assert back.experiment.algorithms[0].config == cfg
    r = back.results[0][0][0]
    assert (r.ics, r.ec, r.sss, r.accuracy) == (0.9, 0.8, 0.7, 1.0)
    assert r.profile.phase_times == prof.phase_times
    assert r.profile.sinkhorn_profiles[0].iteration_count == 20
    assert back.to_dict() == d
