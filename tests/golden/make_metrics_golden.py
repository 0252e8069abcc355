"""Golden values of the reference's alignment metrics (benchmark/experiment.py:115-144).

The metric functions are taken from the reference's source by name (the module
itself imports dataset and plotting dependencies that are not needed here) and
run on small seeded cases; the cases and the reference's outputs are written to
reference_metrics.json next to this script.  Run it where the reference is
checked out:  python tests/golden/make_metrics_golden.py
"""

import ast
import json
import os
from pathlib import Path

import networkx as nx
import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("CUGAL_REFERENCE") or Path(__file__).resolve().parents[3] / "reference")
NAMES = ["edge_correctness", "induced_conserved_structure", "symmetric_substructure", "alignment_accuracy"]


def reference_metrics():
    tree = ast.parse((REF / "benchmark" / "experiment.py").read_text())
    defs = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in NAMES]
    ns = {"np": np}
    exec(compile(ast.Module(body=defs, type_ignores=[]), "experiment.py", "exec"), ns)
    return {name: ns[name] for name in NAMES}


def main():
    fns = reference_metrics()
    cases = []
    rng = np.random.default_rng(0)
    for k, (n, kind) in enumerate([(40, "perm"), (60, "perm"), (60, "noisy"), (50, "dup"), (30, "identity")]):
        g = nx.gnp_random_graph(n, 0.15, seed=k)
        truth = rng.permutation(n)
        h = nx.relabel_nodes(g, {i: int(truth[i]) for i in range(n)})
        h.remove_edges_from(list(h.edges())[: n // 10])
        if kind == "perm":
            answer = rng.permutation(n)
        elif kind == "noisy":
            answer = truth.copy()
            idx = rng.choice(n, 10, replace=False)
            answer[idx] = answer[np.roll(idx, 1)]
        elif kind == "dup":
            answer = truth.copy()
            answer[3] = answer[4]
        else:
            answer = truth.copy()
        A = nx.to_numpy_array(g, nodelist=range(n))
        B = nx.to_numpy_array(h, nodelist=range(n))
        out = {name: float(fns[name](A, B, answer, truth)) for name in NAMES[:3]}
        out["alignment_accuracy"] = float(fns["alignment_accuracy"](truth, answer))
        cases.append({"n": n, "source_edges": [list(map(int, e)) for e in g.edges()],
                      "target_edges": [list(map(int, e)) for e in h.edges()], "answer": answer.tolist(),
                      "truth": truth.tolist(), "reference": out})
    (HERE / "reference_metrics.json").write_text(json.dumps(cases))


if __name__ == "__main__":
    main()
