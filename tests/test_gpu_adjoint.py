"""The device Sinkhorn adjoint (cugal_b200.autograd) against the reference's
solve_log under torch autograd (golden gradients), the FP64 oracle's implicit
adjoint, and finite differences of the FP64 oracle for d objective / d mu."""

from pathlib import Path

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu
GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_adjoint.npz")


def _config(reg, iters=2000, thr=1e-6):
    from cugal_b200.config import Config, SinkhornMethod
    return Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                  sinkhorn_regularization=reg, sinkhorn_iterations=iters, sinkhorn_threshold=thr,
                  sinkhorn_eval_freq=10)


@pytest.mark.parametrize("k", [0, 1])
def test_adjoint_matches_reference_autograd(k):
    from cugal_b200.autograd import sinkhorn_plan
    C0, W, reg = GOLD[f"C{k}"], GOLD[f"W{k}"], float(GOLD[f"reg{k}"])
    C = torch.tensor(C0, dtype=torch.float32, device="cuda", requires_grad=True)
    P = sinkhorn_plan(C, _config(reg))
    np.testing.assert_allclose(P.detach().cpu().numpy(), GOLD[f"P{k}"], rtol=1e-3, atol=1e-5)
    (torch.tensor(W, dtype=torch.float32, device="cuda") * P).sum().backward()
    ref = GOLD[f"dC{k}"]
    np.testing.assert_allclose(C.grad.cpu().numpy(), ref, rtol=1e-3, atol=1e-3 * np.abs(ref).max())


def test_adjoint_matches_oracle_at_scale():
    from cugal_b200.autograd import sinkhorn_adjoint, sinkhorn_plan
    n, reg = 500, 0.05
    rng = np.random.default_rng(9)
    C = torch.tensor(rng.random((n, n)) * 2, dtype=torch.float32, device="cuda")
    W = rng.standard_normal((n, n))
    P = sinkhorn_plan(C, _config(reg, iters=5000, thr=5e-5)).detach()
    dC, iters, rel = sinkhorn_adjoint(P, torch.tensor(W, dtype=torch.float32, device="cuda"), reg)
    assert rel < 1e-6 and iters < 2000
    ref = O.sinkhorn_implicit_adjoint(P.cpu().numpy().astype(np.float64), W, reg)
    np.testing.assert_allclose(dC.cpu().numpy(), ref, rtol=1e-3, atol=1e-4 * np.abs(ref).max())


def _graph_pair(n, seed):
    g = nx.newman_watts_strogatz_graph(n, 6, 0.1, seed=seed)
    h = nx.relabel_nodes(g, dict(zip(range(n), np.random.default_rng(seed).permutation(n).tolist())))
    return g, h


def test_dobjective_dmu_matches_finite_differences():
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.autograd import sinkhorn_plan, structural_objective
    n, reg, mu0, h = 40, 0.2, 0.7, 1e-4
    g, hh = _graph_pair(n, 4)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(hh, "cuda")
    rng = np.random.default_rng(4)
    D = rng.random((n, n)) * 3
    P0 = np.full((n, n), 1.0 / n) + rng.random((n, n)) * 0.01
    Ad = nx.to_numpy_array(g, nodelist=range(n))
    Bd = nx.to_numpy_array(hh, nodelist=range(n))
    base = -2 * Ad @ P0 @ Bd

    def obj64(mu):
        P = O.sinkhorn_plan_log(base + mu * D, reg)
        return -np.sum(P * (Ad @ P @ Bd))

    fd = (obj64(mu0 + h) - obj64(mu0 - h)) / (2 * h)
    mu = torch.tensor(mu0, dtype=torch.float64, device="cuda", requires_grad=True)
    C = torch.tensor(base, dtype=torch.float32, device="cuda") + mu.float() * torch.tensor(D, dtype=torch.float32,
                                                                                           device="cuda")
    P = sinkhorn_plan(C, _config(reg, iters=5000, thr=1e-6))
    structural_objective(P, A, B).backward()
    assert mu.grad.item() == pytest.approx(fd, rel=2e-2, abs=1e-3)


def test_tune_mu_runs_and_descends():
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.autograd import structural_objective, tune_mu, sinkhorn_plan
    n = 300
    g, hh = _graph_pair(n, 5)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(hh, "cuda")
    rng = np.random.default_rng(5)
    D = torch.tensor(rng.random((n, n)) * 3, dtype=torch.float32, device="cuda")
    P0 = torch.full((n, n), 1.0 / n, device="cuda")
    hist = tune_mu(A, B, D, _config(0.05, iters=3000, thr=1e-4), P0, mu0=0.2, steps=5, lr=0.1)
    assert len(hist) == 5
    assert all(np.isfinite(x) for row in hist for x in row)
    assert hist[-1][0] != hist[0][0]
    objs = [row[1] for row in hist]
    assert all(b <= a + 1e-3 * abs(a) for a, b in zip(objs, objs[1:]))  # line search: no increase


@pytest.mark.parametrize("k,every", [(0, 10), (1, 7)])
def test_unrolled_adjoint_matches_reference_autograd(k, every):
    from cugal_b200.autograd import sinkhorn_plan_unrolled
    C0, W, reg = GOLD[f"C{k}"], GOLD[f"W{k}"], float(GOLD[f"reg{k}"])
    C = torch.tensor(C0, dtype=torch.float32, device="cuda", requires_grad=True)
    P = sinkhorn_plan_unrolled(C, _config(reg, iters=300, thr=1e-6), every=every)
    np.testing.assert_allclose(P.detach().cpu().numpy(), GOLD[f"P{k}"], rtol=1e-3, atol=1e-5)
    (torch.tensor(W, dtype=torch.float32, device="cuda") * P).sum().backward()
    ref = GOLD[f"dC{k}"]
    np.testing.assert_allclose(C.grad.cpu().numpy(), ref, rtol=2e-3, atol=2e-3 * np.abs(ref).max())
