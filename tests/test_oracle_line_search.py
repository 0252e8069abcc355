"""The oracle's exact Frank-Wolfe line search (opt-in ``line_search``): the step
rule minimises the parabola on [0, 1], the parabola is the objective exactly
along q - P, and line-search iterates never increase the objective within one
lambda round.  CPU only."""

import networkx as nx
import numpy as np
import pytest
import scipy.sparse

from oracle import fugal_fp64 as O


@pytest.mark.parametrize("seed", range(20))
def test_step_rule_minimises_parabola(seed):
    rng = np.random.default_rng(seed)
    g, Q = rng.standard_normal(2) * 10.0 ** rng.integers(-3, 3, size=2)
    a = O.line_search_alpha(g, Q)
    assert 0.0 <= a <= 1.0
    grid = np.linspace(0.0, 1.0, 2001)
    assert a * g + a * a * Q <= np.min(grid * g + grid * grid * Q) + 1e-12 * (abs(g) + abs(Q))


def test_step_rule_branches():
    assert O.line_search_alpha(-1.0, 2.0) == pytest.approx(0.25)   # interior
    assert O.line_search_alpha(-10.0, 2.0) == 1.0                  # clipped at 1
    assert O.line_search_alpha(1.0, 2.0) == 0.0                    # ascent direction
    assert O.line_search_alpha(-1.0, -2.0) == 1.0                  # concave, descends to 1
    assert O.line_search_alpha(1.0, -0.5) == 0.0                   # concave, f(1) > f(0)
    assert O.line_search_alpha(0.0, 0.0) == 0.0                    # no direction: no step


def _graphs(n, seed):
    g = nx.gnm_random_graph(n, 4 * n, seed=seed)
    h = nx.gnm_random_graph(n, 4 * n, seed=seed + 1)
    A = scipy.sparse.csr_matrix(nx.to_numpy_array(g, nodelist=range(n)))
    B = scipy.sparse.csr_matrix(nx.to_numpy_array(h, nodelist=range(n)))
    return A, B


@pytest.mark.parametrize("lam", [0.0, 2.0])
def test_parabola_is_the_objective(lam):
    n = 40
    A, B = _graphs(n, 3)
    rng = np.random.default_rng(3)
    D = rng.random((n, n))
    P = rng.random((n, n)) / n
    q = rng.random((n, n)) / n
    G = O.sparse_gradient(A, B, P, D, lam)
    _, g, Q = O.line_search_step(A, B, P, G, q, lam)
    f0 = O.fw_objective(A, B, P, D, lam)
    for a in (0.1, 0.5, 1.0):
        fa = O.fw_objective(A, B, P + a * (q - P), D, lam)
        assert fa - f0 == pytest.approx(a * g + a * a * Q, rel=1e-10, abs=1e-10)


def test_gradient_of_objective_is_sparse_gradient():
    n, lam, h = 25, 1.5, 1e-6
    A, B = _graphs(n, 5)
    rng = np.random.default_rng(5)
    D, P = rng.random((n, n)), rng.random((n, n)) / n
    G = O.sparse_gradient(A, B, P, D, lam)
    for i, j in [(0, 0), (3, 17), (24, 2)]:
        E = np.zeros((n, n))
        E[i, j] = h
        fd = (O.fw_objective(A, B, P + E, D, lam) - O.fw_objective(A, B, P - E, D, lam)) / (2 * h)
        assert fd == pytest.approx(G[i, j], rel=1e-6, abs=1e-6)


def test_line_search_objective_non_increasing():
    """Iterate k of a run with k Frank-Wolfe steps (lambda = 0) for k = 1..6: the
    objective never goes up (a = 0 is always admissible)."""
    from cugal_b200.synthetic import noisy_permuted_copy
    n = 50
    g = nx.newman_watts_strogatz_graph(n, 6, 0.1, seed=11)
    h, _ = noisy_permuted_copy(g, np.random.default_rng(11), 3, 3)
    A_csr, B_csr = O.csr_from_graph(g), O.csr_from_graph(h)
    A, B = O.csr_to_scipy(*A_csr, n), O.csr_to_scipy(*B_csr, n)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    D = O.distance_matrix(F1, F2)
    objs, alphas = [O.fw_objective(A, B, np.full((n, n), 1.0 / n), D, 0.0)], None
    for k in range(1, 7):
        tr = O.FWTrace()
        p = O.OracleParams(sinkhorn_regularization=0.5, sinkhorn_method="LOG", sinkhorn_iterations=300,
                           sinkhorn_threshold=1e-6, iter_count=1, frank_wolfe_iter_count=k, line_search=True)
        P = O.find_quasi_permutation_matrix(A_csr, B_csr, D, p, tr)
        objs.append(O.fw_objective(A, B, P, D, 0.0))
        alphas = tr.alphas
    assert all(0.0 <= a <= 1.0 for a in alphas)
    assert all(b <= a + 1e-9 * abs(a) for a, b in zip(objs, objs[1:]))
    assert objs[-1] < objs[0]
