"""Pin the oracle against the reference: golden vectors from the reference's own
Python code (``tests/golden/make_golden.py``) plus networkx / scipy known answers.
CPU only."""

import json
from pathlib import Path

import networkx as nx
import numpy as np
import pytest
import scipy.optimize

from oracle import fugal_fp64 as O

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLD / "reference_golden.npz"))


@pytest.mark.parametrize("name", ["nws16", "ba40", "gaps"])
def test_csr_matches_reference(g, name):
    rp, col = O.csr_from_edges(g[f"csr_{name}_edges"], int(g[f"csr_{name}_n"]))
    assert np.array_equal(rp, g[f"csr_{name}_row_pointers"])
    assert np.array_equal(col, g[f"csr_{name}_col_indices"])


@pytest.mark.parametrize("name", ["nws32", "ba40", "gaps"])
def test_features_match_reference_nx_path(g, name):
    n = int(g[f"feat_{name}_n"])
    rp, col = O.csr_from_edges(g[f"feat_{name}_edges"], n)
    cuda_sem = O.features_cuda_semantics(rp, col)
    ref = g[f"feat_{name}_nx"]
    # degrees are exact; the CUDA-semantics ratios are FP32 of the exact FP64 values
    assert np.array_equal(cuda_sem[:, 0], ref[:, 0].astype(np.float32))
    np.testing.assert_allclose(cuda_sem, ref, rtol=2e-7, atol=1e-7)


def test_triangle_counts_known_answer():
    graph = nx.newman_watts_strogatz_graph(200, 8, 0.2, seed=3)
    rp, col = O.csr_from_graph(graph)
    deg, tri = O.triangle_counts(rp, col)
    tri_nx = nx.triangles(graph)
    assert all(tri[v] == 2 * tri_nx[v] for v in range(200))
    assert all(deg[v] == graph.degree(v) for v in range(200))


def test_distance_matches_reference(g):
    D = O.distance_matrix(g["dist_F1"], g["dist_F2"])
    np.testing.assert_allclose(D, g["dist_D"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("lam", [0, 3])
def test_dense_gradient_matches_reference(g, lam):
    G = O.dense_gradient(g["grad_A"], g["grad_B"], g["grad_P"], g["grad_D"], lam, double_lambda=True)
    np.testing.assert_allclose(G, g[f"grad_dense_l{lam}"], rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("lam", [0, 3])
def test_sparse_gradient_is_dense_with_single_lambda(g, lam):
    A, B = g["grad_A"], g["grad_B"]
    rpa, cola = O.csr_from_edges(np.argwhere(np.triu(A) > 0), len(A))
    rpb, colb = O.csr_from_edges(np.argwhere(np.triu(B) > 0), len(B))
    Gs = O.sparse_gradient(O.csr_to_scipy(rpa, cola, len(A)), O.csr_to_scipy(rpb, colb, len(B)),
                           g["grad_P"], g["grad_D"], lam)
    Gd = O.dense_gradient(A, B, g["grad_P"], g["grad_D"], lam, double_lambda=False)
    np.testing.assert_allclose(Gs, Gd, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", ["log_patched", "log_mutating", "log_momentum", "log_momentum_neg", "std"])
def test_sinkhorn_matches_reference(g, case):
    reg, thr, freq, mstart = g[f"sk_{case}_params"]
    freq = int(freq)
    mstart = None if mstart < 0 else int(mstart)
    n = g["sk_C"].shape[0]
    solve = O.sinkhorn_standard_solve if case == "std" else O.sinkhorn_log_solve
    kw = {} if case == "std" else {"mutating_marginal": case == "log_mutating"}
    u0 = np.full(n, 1.0 / n) if case == "std" else np.zeros(n)
    r1 = solve(g["sk_C"], u0, u0.copy(), reg, 200, thr, freq, mstart, **kw)
    assert r1.iteration_count == int(g[f"sk_{case}_it1"])
    np.testing.assert_allclose(r1.errors, g[f"sk_{case}_err1"], rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(r1.u, g[f"sk_{case}_u1"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(r1.v, g[f"sk_{case}_v1"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(r1.K, g[f"sk_{case}_K1"], rtol=1e-11, atol=1e-11)
    r2 = solve(g[f"sk_{case}_C2"], r1.u, r1.v, reg, 200, thr, freq, mstart, **kw)
    assert r2.iteration_count == int(g[f"sk_{case}_it2"])
    np.testing.assert_allclose(r2.u, g[f"sk_{case}_u2"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(r2.v, g[f"sk_{case}_v2"], rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("name,log", [("log", True), ("std", False)])
def test_update_matches_reference(g, name, log):
    P = g["upd_P"].copy()
    diff = O.update_quasi_permutation(P, g["upd_K"].copy(), g["upd_u"], g["upd_v"], 0.4, log)
    np.testing.assert_allclose(P, g[f"upd_{name}_P"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(diff, g[f"upd_{name}_q"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("method", ["GREEDY", "DOUBLE_GREEDY", "PARALLEL_GREEDY", "RAND", "MORE_RAND"])
def test_greedy_lap_matches_reference(g, method):
    P = g["lap_P"].copy()
    kw = {}
    if method in ("RAND", "MORE_RAND"):
        kw["order"] = g[f"lap_{method}_order"]
    if method == "MORE_RAND":
        kw["uniforms"] = g["lap_MORE_RAND_uniforms"]
    cols = O.greedy_lap(P, method, **kw)
    assert np.array_equal(cols, g[f"lap_{method}_cols"])
    assert np.array_equal(P, g[f"lap_{method}_P"])


def test_scipy_lap_is_a_maximum_assignment(g):
    P = g["lap_P"]
    cols = O.hungarian(P.copy(), "SCIPY")
    assert sorted(cols) == list(range(len(P)))
    _, ref = scipy.optimize.linear_sum_assignment(P, maximize=True)
    assert np.isclose(P[np.arange(len(P)), cols].sum(), P[np.arange(len(P)), ref].sum())


@pytest.mark.parametrize("name,mutating,lap", [("patched_scipy", False, "SCIPY"),
                                               ("patched_dgreedy", False, "DOUBLE_GREEDY"),
                                               ("mutating_scipy", True, "SCIPY")])
def test_full_alignment_matches_reference(g, name, mutating, lap):
    src = nx.Graph()
    src.add_nodes_from(range(40))
    src.add_edges_from(g["e2e_src_edges"].tolist())
    tgt = nx.Graph()
    tgt.add_nodes_from(range(40))
    tgt.add_edges_from(g["e2e_tgt_edges"].tolist())
    p = O.OracleParams(sinkhorn_regularization=0.05, sinkhorn_method="LOG", sinkhorn_iterations=200,
                       sinkhorn_threshold=1e-6, sinkhorn_eval_freq=10, mu=1.0, iter_count=3,
                       frank_wolfe_iter_count=10, use_sparse_adjacency=False, hungarian_method=lap,
                       mutating_marginal=mutating, double_lambda=True)
    trace = O.FWTrace()
    P, mapping, sp = O.cugal(src, tgt, p, features="nx", trace=trace)
    assert trace.sinkhorn_iterations == list(g[f"e2e_{name}_sk_iters"])
    assert trace.frank_wolfe_iterations == int(g[f"e2e_{name}_fw"])
    np.testing.assert_allclose(P, g[f"e2e_{name}_P"], rtol=1e-8, atol=1e-10)
    assert [m[1] for m in mapping] == list(g[f"e2e_{name}_cols"])
    assert np.isclose(sp, float(g[f"e2e_{name}_sparsity"]))


def test_lehmann_momentum_negative_index():
    # index = 10 // 10 = 1 -> errors[0] / errors[-1] (Python negative index)
    errs = [0.5, 0.25, 0.2]
    w = O.lehmann_momentum(errs, 10, 10)
    ratio = min(errs[0] / errs[-1], 0.99)
    assert w == pytest.approx(2.0 / (1.0 + (1 - ratio ** 0.1) ** 0.5))
    assert O.lehmann_momentum(errs, None, 10) == 1.0
    assert O.lehmann_momentum([0.1], 50, 10) == 1.0


def test_config_dicts_roundtrip():
    from cugal_b200.config import Config
    for d in json.loads((GOLD / "reference_configs.json").read_text()):
        c = Config.from_dict(dict(d))
        back = c.to_dict()
        for k, v in d.items():
            assert back[k] == v, k
