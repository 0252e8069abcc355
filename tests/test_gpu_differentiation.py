"""The Sinkhorn adjoint on the differentiation workload: Newman-Watts-Strogatz
n=4096 (k 12, p 0.05, seed 3, 3% edge noise), C(mu) = -2 A P0 B + mu D at the
uniform P0 with D the feature distance, log Sinkhorn reg 0.05, and the
structural objective L = -<P, A P B> at the converged plan.

* dL/dmu from this path (FP32 forward to the 1e-6 marginal tolerance, implicit
  adjoint on the device) against FP64 central differences with step 1e-6
  (oracle/fugal_torch64.py solves, converged to 1e-12), and against torch
  autograd in FP64 through the reference's solve_log iteration
  (cugal/sinkhorn.py:99-116, oracle/fugal_torch64.solve_log_differentiable);
* dL/dC elementwise against the same autograd gradient.

reg 0.05 rather than the alignment's 1e-3: at 1e-3 the converged plan is a
near-hard assignment and L is piecewise constant in mu at this scale, so
derivatives exist only in a tiny neighbourhood."""

import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu

REG, MU0, H = 0.05, 0.2, 1e-6


def _workload():
    import networkx as nx
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config
    from cugal_b200.feature_extraction import Features
    from cugal_b200.synthetic import make_pair
    src, tgt, _, _ = make_pair("nws4096")
    n = src.number_of_nodes()
    A, B = Adjacency.from_graph(src, "cuda"), Adjacency.from_graph(tgt, "cuda")
    D = Features.create(A, B, Config(device="cuda", dtype=torch.float32, mu=1.0)).distance_matrix()[:n, :n]
    Ad = torch.tensor(nx.to_numpy_array(src, nodelist=range(n)), dtype=torch.float64, device="cuda")
    Bd = torch.tensor(nx.to_numpy_array(tgt, nodelist=range(n)), dtype=torch.float64, device="cuda")
    # A P0 B at the uniform P0 = 1/n: the outer product of the degree vectors over n
    base = -2.0 * torch.outer(Ad.sum(1), Bd.sum(0)) / n
    return n, A, B, Ad, Bd, D.contiguous(), base


def _objective64(P, Ad, Bd):
    return -(P * (Ad @ P @ Bd)).sum()


def _solve64(C, u=None, v=None, threshold=1e-12):
    from oracle import fugal_torch64 as T
    n = C.shape[0]
    K = -C / REG
    u = torch.zeros(n, dtype=torch.float64, device="cuda") if u is None else u.clone()
    v = torch.zeros(n, dtype=torch.float64, device="cuda") if v is None else v.clone()
    rec = T.sinkhorn_log_solve_(K, u, v, 20000, threshold, 10, block=1024)
    return torch.exp(K + u[:, None] + v[None, :]), u, v, rec.iterations


def test_nws4096_mu_gradient_against_fp64_differences_and_reference_autograd():
    from cugal_b200.autograd import sinkhorn_plan, structural_objective
    from cugal_b200.config import Config, SinkhornMethod
    from oracle import fugal_torch64 as T
    n, A, B, Ad, Bd, D, base = _workload()
    D64 = D.double()
    # this path: FP32 forward, device adjoint
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, sinkhorn_regularization=REG,
                 sinkhorn_iterations=20000, sinkhorn_threshold=1e-6, sinkhorn_eval_freq=10)
    mu = torch.tensor(MU0, dtype=torch.float64, device="cuda", requires_grad=True)
    C = (base.float() + mu.float() * D)
    C.retain_grad()
    L = structural_objective(sinkhorn_plan(C, cfg), A, B)
    L.backward()
    g_ours = float(mu.grad.item())
    dC_ours = C.grad.double()
    # FP64 central differences, step 1e-6, from converged FP64 solves
    P0, u0, v0, it0 = _solve64(base + MU0 * D64)
    Lp = float(_objective64(_solve64(base + (MU0 + H) * D64, u0, v0)[0], Ad, Bd).item())
    Lm = float(_objective64(_solve64(base + (MU0 - H) * D64, u0, v0)[0], Ad, Bd).item())
    fd = (Lp - Lm) / (2 * H)
    # torch autograd in FP64 through the reference's iteration, run as long as the FP64 solve took
    C64 = (base + MU0 * D64).requires_grad_(True)
    P_ad = T.solve_log_differentiable(C64, REG, it0)
    _objective64(P_ad, Ad, Bd).backward()
    dC_ref = C64.grad
    g_ref = float((dC_ref * D64).sum().item())
    print(f"\n[nws4096 reg {REG} mu {MU0}] dL/dmu: adjoint {g_ours:.6e}, FP64 central difference (h {H:g}) {fd:.6e}, "
          f"autograd through solve_log {g_ref:.6e}; FP64 solve {it0} iterations; "
          f"max|dC - dC_ref| / max|dC_ref| = {float((dC_ours - dC_ref).abs().max() / dC_ref.abs().max()):.2e}")
    assert g_ref == pytest.approx(fd, rel=1e-5, abs=1e-9)
    assert g_ours == pytest.approx(fd, rel=1e-3, abs=1e-6)
    torch.testing.assert_close(dC_ours, dC_ref, rtol=1e-2, atol=1e-3 * float(dC_ref.abs().max()))
