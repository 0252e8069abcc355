"""Alignment metrics (EC, ICS, S3, accuracy) against the reference's own
functions' outputs (tests/golden/reference_metrics.json, written by
tests/golden/make_metrics_golden.py): the oracle on CPU, the device overlap
count on the GPU."""

import json
from pathlib import Path

import networkx as nx
import numpy as np
import pytest

from oracle import fugal_fp64 as O

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "reference_metrics.json").read_text())


def _dense(case, key):
    g = nx.Graph()
    g.add_nodes_from(range(case["n"]))
    g.add_edges_from(map(tuple, case[key]))
    return g, nx.to_numpy_array(g, nodelist=range(case["n"]))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_oracle_metrics_match_reference(k):
    c = CASES[k]
    _, A = _dense(c, "source_edges")
    _, B = _dense(c, "target_edges")
    ref = c["reference"]
    assert O.edge_correctness(A, B, c["answer"], c["truth"]) == pytest.approx(ref["edge_correctness"], abs=0)
    assert O.induced_conserved_structure(A, B, c["answer"], c["truth"]) == pytest.approx(
        ref["induced_conserved_structure"], abs=0)
    assert O.symmetric_substructure(A, B, c["answer"], c["truth"]) == pytest.approx(
        ref["symmetric_substructure"], abs=0)


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(CASES)))
def test_device_metrics_match_reference(k):
    from cugal_b200 import metrics
    from cugal_b200.adjacency import Adjacency
    c = CASES[k]
    g, _ = _dense(c, "source_edges")
    h, _ = _dense(c, "target_edges")
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    res = metrics.Result.calculate(None, A, B, np.array(c["answer"]), np.array(c["truth"]))
    ref = c["reference"]
    assert res.ec == ref["edge_correctness"]
    assert res.ics == ref["induced_conserved_structure"]
    assert res.sss == ref["symmetric_substructure"]
    assert res.accuracy == ref["alignment_accuracy"]


@pytest.mark.gpu
def test_device_overlap_large_graph_matches_oracle():
    from cugal_b200 import metrics
    from cugal_b200.adjacency import Adjacency
    n = 3000
    rng = np.random.default_rng(5)
    g = nx.barabasi_albert_graph(n, 4, seed=5)
    truth = rng.permutation(n)
    h = nx.relabel_nodes(g, {i: int(truth[i]) for i in range(n)})
    answer = truth.copy()
    idx = rng.choice(n, 300, replace=False)
    answer[idx] = answer[rng.permutation(idx)]
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    got = metrics.overlap(A, B, answer, truth)
    Ad = nx.to_numpy_array(g, nodelist=range(n))
    Bd = nx.to_numpy_array(h, nodelist=range(n))
    assert got == O.alignment_overlap(Ad, Bd, answer, truth)


@pytest.mark.parametrize("seed", [0, 1])
def test_edge_array_matches_edge_list(seed):
    """The adjacency-walk edge extraction gives the same directed pairs as
    graph.edges() plus reversals, self-loops included (CPU)."""
    from cugal_b200.adjacency import edge_array
    g = nx.gnm_random_graph(300, 1200, seed=seed)
    g.add_edges_from([(5, 5), (17, 17)])
    got = edge_array(g)
    flat = np.array([e for e in g.edges()], dtype=np.int64)
    want = np.concatenate([flat, flat[:, ::-1]])
    assert got.dtype == np.int32 and got.shape == want.shape
    key = lambda a: np.lexsort((a[:, 1], a[:, 0]))
    np.testing.assert_array_equal(got[key(got)], want[key(want)].astype(np.int32))
