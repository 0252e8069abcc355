"""The torch FP64 restatement (oracle/fugal_torch64.py, used on the GPU for the
large workloads) against the numpy FP64 oracle, on the CPU."""

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O
from oracle import fugal_torch64 as T


def pair(n, seed):
    from cugal_b200.synthetic import noisy_permuted_copy
    g = nx.newman_watts_strogatz_graph(n, 6, 0.1, seed=seed)
    h, perm = noisy_permuted_copy(g, np.random.default_rng(seed), 3, 3)
    return g, h, perm


@pytest.mark.parametrize("lam_scale,reg", [(1.0, 0.05), (2.0, 0.02)])
def test_torch64_loop_matches_numpy_oracle(lam_scale, reg):
    g, h, _ = pair(60, 3)
    A_csr, B_csr = O.csr_from_graph(g), O.csr_from_graph(h)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    p = O.OracleParams(sinkhorn_regularization=reg, sinkhorn_iterations=300, sinkhorn_threshold=1e-6,
                       sinkhorn_eval_freq=10, mu=1.0, iter_count=3, frank_wolfe_iter_count=5,
                       use_sparse_adjacency=lam_scale == 1.0, double_lambda=True)
    tr = O.FWTrace()
    P_ref = O.find_quasi_permutation_matrix(A_csr, B_csr, O.distance_matrix(F1, F2), p, tr)
    tt = T.Trace()
    P = T.find_quasi_permutation_matrix(A_csr, B_csr, F1, F2, reg=reg, iter_count=3, fw_iter_count=5,
                                        sinkhorn_iterations=300, threshold=1e-6, eval_freq=10, mu=1.0,
                                        lam_scale=lam_scale, device="cpu", block=16, trace=tt)
    assert tt.sinkhorn_iterations == tr.sinkhorn_iterations
    np.testing.assert_allclose(P.numpy(), P_ref, rtol=0, atol=1e-10)
    np.testing.assert_allclose(tt.gaps, tr.gaps, rtol=1e-8, atol=1e-10)


def test_torch64_truncated_run_and_objective():
    g, h, perm = pair(48, 4)
    A_csr, B_csr = O.csr_from_graph(g), O.csr_from_graph(h)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    kw = dict(reg=0.05, iter_count=2, fw_iter_count=4, sinkhorn_iterations=200, threshold=1e-6, eval_freq=10,
              device="cpu", block=7)
    tt = T.Trace()
    P3 = T.find_quasi_permutation_matrix(A_csr, B_csr, F1, F2, max_steps=3, trace=tt, objective_every=True, **kw)
    assert len(tt.sinkhorn_iterations) == 3 and len(tt.objectives) == 3
    p = O.OracleParams(sinkhorn_regularization=0.05, sinkhorn_iterations=200, sinkhorn_threshold=1e-6,
                       sinkhorn_eval_freq=10, mu=1.0, iter_count=1, frank_wolfe_iter_count=3)
    P_ref = O.find_quasi_permutation_matrix(A_csr, B_csr, O.distance_matrix(F1, F2), p)
    np.testing.assert_allclose(P3.numpy(), P_ref, rtol=0, atol=1e-10)
    A = O.csr_to_scipy(*A_csr, 48)
    B = O.csr_to_scipy(*B_csr, 48)
    ref_obj = O.fw_objective(A, B, P_ref, O.distance_matrix(F1, F2), 0.0)
    assert tt.objectives[-1] == pytest.approx(ref_obj, rel=1e-12, abs=1e-12)
    cols = T.double_greedy(torch.as_tensor(P_ref))
    assert np.array_equal(cols, O.greedy_lap(P_ref.copy(), "DOUBLE_GREEDY"))
