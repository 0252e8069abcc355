"""GPU parity: CSR construction, features, adjacency products, greedy rounding.
Integer results and index results are compared bit-exactly with the oracle."""

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu


def graphs():
    g_gaps = nx.Graph([(1, 3), (3, 5), (5, 9), (2, 3), (9, 2)])
    g_gaps.add_nodes_from(range(12))  # nodes 0, 4, 6, 7, 8, 10, 11 isolated (incl. both ends)
    star = nx.star_graph(5000)  # one row of 5000 columns (sorted in shared memory)
    return {
        "nws32": nx.newman_watts_strogatz_graph(32, 10, 0.1, seed=1),
        "ba3000": nx.barabasi_albert_graph(3000, 5, seed=2),
        "er2000": nx.fast_gnp_random_graph(2000, 0.01, seed=3),
        "gaps": g_gaps,
        "edgeless": nx.empty_graph(10),
        "star": star,
        "k40": nx.complete_graph(40),
    }


@pytest.mark.parametrize("name", list(graphs()))
def test_csr_and_features_bit_exact(name):
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.feature_extraction import average_neighbor_features, graph_features
    g = graphs()[name]
    rp, col = O.csr_from_graph(g)
    A = Adjacency.from_graph(g, "cuda")
    assert np.array_equal(A.row_pointers.cpu().numpy(), rp)
    assert np.array_equal(A.col_indices.cpu().numpy(), col)
    deg, clust, dc, tc = graph_features(A, with_counts=True)
    odeg, otri = O.triangle_counts(rp, col)
    assert np.array_equal(dc.cpu().numpy(), odeg)
    assert np.array_equal(tc.cpu().numpy(), otri)
    if name in ("nws32", "k40"):
        tri_nx = nx.triangles(g)
        assert all(otri[v] == 2 * tri_nx[v] for v in g.nodes)
    oclust = O.clustering_from_counts(odeg, otri)
    assert np.array_equal(clust.cpu().numpy(), oclust)
    assert np.array_equal(deg.cpu().numpy(), odeg.astype(np.float32))
    for vals in (deg, clust):
        avg = average_neighbor_features(A, vals).cpu().numpy()
        assert np.array_equal(avg, O.average_neighbor(rp, col, vals.cpu().numpy()))


@pytest.mark.parametrize("workload", ["ba8192", "er32768"])
def test_workload_degrees_and_triangles_bit_exact(workload):
    """Degrees, triangle counts, clustering and neighbour averages of both graphs
    of the Barabasi-Albert n=8192 (m=5, seed 1, 5% noise) and Erdos-Renyi
    n=32768 (mean degree 16, seed 2, 2% noise) workloads, bit for bit."""
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.feature_extraction import average_neighbor_features, graph_features
    from cugal_b200.synthetic import make_pair
    src, tgt, _, _ = make_pair(workload)
    for g in (src, tgt):
        rp, col = O.csr_from_graph(g)
        A = Adjacency.from_graph(g, "cuda")
        assert np.array_equal(A.row_pointers.cpu().numpy(), rp)
        assert np.array_equal(A.col_indices.cpu().numpy(), col)
        deg, clust, dc, tc = graph_features(A, with_counts=True)
        odeg, otri = O.triangle_counts(rp, col)
        assert np.array_equal(dc.cpu().numpy(), odeg)
        assert np.array_equal(tc.cpu().numpy(), otri)
        assert np.array_equal(clust.cpu().numpy(), O.clustering_from_counts(odeg, otri))
        for vals in (deg, clust):
            avg = average_neighbor_features(A, vals).cpu().numpy()
            assert np.array_equal(avg, O.average_neighbor(rp, col, vals.cpu().numpy()))


def test_features_match_reference_nx_path_within_fp32():
    from cugal_b200.config import Config
    from cugal_b200.feature_extraction import extract_features_cuda
    g = nx.newman_watts_strogatz_graph(32, 10, 0.1, seed=13)
    ours = extract_features_cuda(g, Config(device="cuda", dtype=torch.float32)).cpu().numpy()
    np.testing.assert_allclose(ours, O.features_nx_semantics(g), rtol=2e-7, atol=1e-7)


def test_create_adjacency_from_unsorted_directed_pairs():
    from cugal_b200 import cuda_kernels as ck
    rng = np.random.default_rng(0)
    n = 500
    pairs = rng.integers(0, n, size=(3000, 2)).astype(np.int32)
    edges = torch.tensor(pairs.reshape(-1), device="cuda")
    col = torch.empty(3000, dtype=torch.int32, device="cuda")
    rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    ck.create_adjacency(edges, col, rp)
    # row y receives column x (Edge{col, row} packing of cuda_kernels/adjacency.cu)
    erp, ecol = O.csr_from_edges(pairs[:, ::-1], n, undirected=False)
    assert np.array_equal(rp.cpu().numpy(), erp)
    assert np.array_equal(col.cpu().numpy(), ecol)


@pytest.mark.parametrize("n", [8, 129, 300])
def test_adjacency_matmul_matches_dense(n):
    from cugal_b200.adjacency import Adjacency
    rng = np.random.default_rng(n)
    dense = (rng.random((n, n)) < 0.05).astype(np.float32)
    A = Adjacency.from_dense(torch.tensor(dense, device="cuda"))
    M = torch.tensor(rng.standard_normal((n, n)), dtype=torch.float32, device="cuda")
    np.testing.assert_allclose(A.mul(M).cpu().numpy(), dense @ M.cpu().numpy(), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(A.mul(M, negate_lhs=True).cpu().numpy(), -(dense @ M.cpu().numpy()),
                               rtol=1e-5, atol=1e-5)
    MT = M.t()
    out = A.mul(MT)
    np.testing.assert_allclose(out.cpu().numpy(), dense @ MT.cpu().numpy(), rtol=1e-5, atol=1e-5)


def _lap_matrix(n, seed, zero_rows=0, ties=False):
    rng = np.random.default_rng(seed)
    P = (rng.random((n, n)) ** 6).astype(np.float32)
    for r in range(zero_rows):
        P[(r * 7) % n] = 0.0
    if ties:
        P[5] = P[9]
        P[11, :] = 0.25
    return P


@pytest.mark.parametrize("method", ["GREEDY", "DOUBLE_GREEDY", "PARALLEL_GREEDY", "RAND"])
@pytest.mark.parametrize("k", [1, 2, 8, 16])
@pytest.mark.parametrize("case", ["plain", "zeros", "ties"])
def test_greedy_rounding_bit_exact(method, k, case):
    from cugal_b200.config import HungarianMethod
    from cugal_b200.greedy_lap import greedy_assign
    n = 300
    P = _lap_matrix(n, 7, zero_rows=20 if case == "zeros" else 0, ties=case == "ties")
    if method == "PARALLEL_GREEDY":
        idx = np.arange(0, n, 3)
        P[idx, (idx * 5) % n] = 0.75
    order = np.random.default_rng(3).permutation(n) if method == "RAND" else None
    Pg = torch.tensor(P, device="cuda")
    cols = greedy_assign(Pg, HungarianMethod[method], candidates=k, mutate=True,
                         order=None if order is None else torch.tensor(order)).cpu().numpy()
    Po = P.copy()
    ref = O.greedy_lap(Po, method, order=order)
    assert np.array_equal(cols, ref)
    assert np.array_equal(Pg.cpu().numpy(), Po)


def test_greedy_rounding_against_reference_golden():
    from pathlib import Path
    from cugal_b200.config import HungarianMethod
    from cugal_b200.greedy_lap import greedy_assign
    g = dict(np.load(Path(__file__).resolve().parent / "golden" / "reference_golden.npz"))
    for method in ["GREEDY", "DOUBLE_GREEDY", "PARALLEL_GREEDY", "RAND"]:
        Pg = torch.tensor(g["lap_P"], dtype=torch.float32, device="cuda")
        # the reference ran on float64; the matrix has no ties, so the FP32 order is the same
        order = torch.tensor(g["lap_RAND_order"]) if method == "RAND" else None
        cols = greedy_assign(Pg, HungarianMethod[method], candidates=4, order=order).cpu().numpy()
        assert np.array_equal(cols, g[f"lap_{method}_cols"]), method


def test_count_le_matches_numpy():
    from cugal_b200 import _native as N
    P = torch.rand((333, 333), device="cuda") ** 8
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    eps = float(torch.finfo(torch.float32).eps)
    N.call("fugal_count_le", P.data_ptr(), 333, 333, eps, cnt.data_ptr(), N.stream_handle())
    assert int(cnt.item()) == int((P.cpu().numpy() <= eps).sum())


@pytest.mark.parametrize("n,case", [(300, "plain"), (300, "zeros"), (1000, "plain"), (70, "ties")])
def test_more_rand_rounding_matches_oracle(n, case):
    """MORE_RAND (cugal/greedy_lap.py:34-48) with given row order and draws: the
    same columns and the same mutated P as the oracle."""
    from cugal_b200.greedy_lap import sampled_assign
    P = _lap_matrix(n, 9, zero_rows=n // 10 if case == "zeros" else 0, ties=case == "ties")
    rng = np.random.default_rng(4)
    order = rng.permutation(n)
    uniforms = rng.random(n)
    Pg = torch.tensor(P, device="cuda")
    cols = sampled_assign(Pg, torch.tensor(order), uniforms).cpu().numpy()
    Po = P.astype(np.float64)
    ref = O.greedy_lap(Po, "MORE_RAND", order=order, uniforms=uniforms)
    assert np.array_equal(cols, ref)
    assert np.array_equal(Pg.cpu().numpy(), Po.astype(np.float32))


def test_more_rand_against_reference_golden():
    from pathlib import Path
    from cugal_b200.greedy_lap import sampled_assign
    g = dict(np.load(Path(__file__).resolve().parent / "golden" / "reference_golden.npz"))
    Pg = torch.tensor(g["lap_P"], dtype=torch.float32, device="cuda")
    cols = sampled_assign(Pg, torch.tensor(g["lap_MORE_RAND_order"]), g["lap_MORE_RAND_uniforms"]).cpu().numpy()
    assert np.array_equal(cols, g["lap_MORE_RAND_cols"])
    np.testing.assert_allclose(Pg.cpu().numpy(), g["lap_MORE_RAND_P"], rtol=1e-6, atol=0)
