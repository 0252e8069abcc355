"""Scaling-form Sinkhorn (SinkhornMethod.STANDARD) on the device against the FP64
oracle (cugal/sinkhorn.py:122-144, cugal/pred.py:77-86,136-141): the solve
(iteration count, error sequence, scaling vectors), the update with its gap, and
a whole alignment with the STANDARD method."""

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu


def _problem(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.random((n, n)) * 3.0).astype(np.float32)


@pytest.mark.parametrize("n,mstart", [(64, None), (300, None), (300, 20), (1000, None)])
def test_standard_solve_matches_oracle(n, mstart):
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.sinkhorn import SinkhornState
    from cugal_b200.profile import SinkhornProfile
    C = _problem(n, n)
    reg, thr = 0.5, 1e-4
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.STANDARD,
                 sinkhorn_regularization=reg, sinkhorn_iterations=300, sinkhorn_threshold=thr,
                 sinkhorn_eval_freq=10, sinkhorn_momentum_start=mstart)
    state = SinkhornState(n, cfg)
    prof = SinkhornProfile()
    K, u, v = state.solve(torch.tensor(C, device="cuda"), cfg, prof)
    ref = O.sinkhorn_standard_solve(C.astype(np.float64), np.full(n, 1.0 / n), np.full(n, 1.0 / n), reg, 300, thr,
                                    10, mstart)
    assert prof.iteration_count == ref.iteration_count
    np.testing.assert_allclose(prof.errors, ref.errors, rtol=2e-3, atol=2e-6 * n)
    np.testing.assert_allclose(u.cpu().numpy(), ref.u, rtol=1e-3)
    np.testing.assert_allclose(v.cpu().numpy(), ref.v, rtol=1e-3)
    np.testing.assert_allclose(K.cpu().numpy(), ref.K, rtol=1e-6, atol=1e-30)


def test_standard_update_matches_oracle():
    from cugal_b200 import _native as N
    n = 200
    rng = np.random.default_rng(3)
    C = (rng.random((n, n)) * 2).astype(np.float32)
    K = np.exp(-C / 0.5).astype(np.float32)
    u = (rng.random(n) + 0.5).astype(np.float32)
    v = (rng.random(n) + 0.5).astype(np.float32)
    P = (rng.random((n, n)) / n).astype(np.float32)
    t = {k: torch.tensor(x, device="cuda") for k, x in dict(C=C, K=K, u=u, v=v, P=P).items()}
    gap = torch.zeros(1, dtype=torch.float64, device="cuda")
    N.call("fugal_fw_update_standard", n, t["P"].data_ptr(), n, t["K"].data_ptr(), n, t["u"].data_ptr(),
           t["v"].data_ptr(), t["C"].data_ptr(), n, 0.4, gap.data_ptr(), N.stream_handle(torch.device("cuda")))
    Pr = P.astype(np.float64)
    step = O.update_quasi_permutation(Pr, K.astype(np.float64), u.astype(np.float64), v.astype(np.float64), 0.4,
                                      log=False)
    np.testing.assert_allclose(t["P"].cpu().numpy(), Pr, rtol=1e-5, atol=1e-7)
    ref_gap = float(np.sum(C.astype(np.float64) * step / 0.4))
    assert abs(gap.item() - ref_gap) <= 1e-4 * abs(ref_gap) + 1e-6


def test_full_alignment_standard_matches_oracle():
    from cugal_b200 import Config, HungarianMethod, Profile, SinkhornMethod, cugal
    n = 60
    rng = np.random.default_rng(7)
    g = nx.newman_watts_strogatz_graph(n, 6, 0.2, seed=7)
    h = nx.relabel_nodes(g, dict(zip(range(n), rng.permutation(n).tolist())))
    params = dict(sinkhorn_regularization=0.5, sinkhorn_iterations=200, sinkhorn_threshold=1e-4,
                  sinkhorn_eval_freq=10, mu=1.0, iter_count=2, frank_wolfe_iter_count=5)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.STANDARD,
                 use_sparse_adjacency=True, hungarian_method=HungarianMethod.SCIPY, **params)
    prof = Profile()
    P, mapping = cugal(nx.Graph(g), nx.Graph(h), cfg, prof)
    trace = O.FWTrace()
    Pr, mref, _ = O.cugal(nx.Graph(g), nx.Graph(h),
                          O.OracleParams(sinkhorn_method="STANDARD", use_sparse_adjacency=True,
                                         hungarian_method="SCIPY", **params), features="cuda", trace=trace)
    assert prof.frank_wolfe_iterations == trace.frank_wolfe_iterations == 10
    its = [p.iteration_count for p in prof.sinkhorn_profiles]
    assert max(abs(a - b) for a, b in zip(its, trace.sinkhorn_iterations)) <= 10
    np.testing.assert_allclose(P, Pr, atol=1e-3)
    assert [m[1] for m in mapping] == [m[1] for m in mref]
