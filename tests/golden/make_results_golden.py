"""A sample of the reference's own result files (benchmark/results/*.json,
written by benchmark/experiment.py:513-555) for the result-file round-trip test.

Two files are sampled: one run with the sparse GPU path (per-solve Sinkhorn
profiles) and one with FUGAL's own configuration; long lists (Sinkhorn profiles,
their error lists, graphs, noise levels, runs) are cut to their first few
entries so that the fixture stays small.  Run it where the reference is checked
out:  python tests/golden/make_results_golden.py
"""

import json
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("CUGAL_REFERENCE") or Path(__file__).resolve().parents[3] / "reference") / "benchmark" / "results"
FILES = ["CUGAL_res.json", "FUGAL_res2.json"]


def trim(d: dict, k: int = 2) -> dict:
    exp = d["experiment"]
    n_graphs, n_levels = min(k, len(exp["graphs"])), min(k, len(exp["noise_levels"]))
    exp = dict(exp, graphs=exp["graphs"][:n_graphs], noise_levels=exp["noise_levels"][:n_levels])
    results = []
    for per_graph in d["results"][:n_graphs]:
        rows = []
        for per_level in per_graph[:n_levels]:
            cell = []
            for r in per_level:
                prof = dict(r["profile"])
                prof["sinkhorn_profiles"] = [dict(sp, errors=sp["errors"][:3]) for sp in prof["sinkhorn_profiles"][:3]]
                cell.append(dict(r, profile=prof))
            rows.append(cell)
        results.append(rows)
    return dict(d, experiment=exp, results=results)


def main():
    out = {name: trim(json.loads((REF / name).read_text())) for name in FILES}
    (HERE / "reference_results_sample.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
