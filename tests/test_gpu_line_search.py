"""GPU parity of the exact Frank-Wolfe line search (``Config.line_search``)
against the FP64 oracle: the three device sums g = <G, d>, <d, d>, <d, W>, the
step rule on each of its branches, the update of P, and whole alignments.

Tolerances: sums within 1e-5 of the sum of absolute terms (FP32 direction and
SpMM, FP64 accumulation); the device step equals the rule applied to the device
sums to 1e-12 and the oracle's step to 1e-4 when interior; P within 1e-6 of
P0 + a d."""

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu


def _inputs(n, seed, standard):
    from cugal_b200.adjacency import Adjacency
    rng = np.random.default_rng(seed)
    g = nx.gnm_random_graph(n, 5 * n, seed=seed)
    h = nx.gnm_random_graph(n, 5 * n, seed=seed + 1)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    ld = (n + 3) // 4 * 4
    dev = "cuda"

    def mat(x):
        t = torch.zeros((n, ld), dtype=torch.float32, device=dev)
        t[:, :n] = torch.tensor(x, dtype=torch.float32)
        return t

    P = mat(rng.random((n, n)) / n)
    if standard:
        # q = (K v) u with K = exp(-C): large where C is small, so the direction descends
        C0 = rng.random((n, n)) * 4
        C = mat(C0)
        K = mat(np.exp(-C0))
        u = torch.tensor(2 / np.sqrt(n) * (1 + 0.1 * rng.standard_normal(n)), dtype=torch.float32, device=dev)
        v = torch.tensor(2 / np.sqrt(n) * (1 + 0.1 * rng.standard_normal(n)), dtype=torch.float32, device=dev)
        U = V = None
    else:
        # large L -> large q and small G, so the direction descends
        C = mat(-rng.random((n, n)) * 6)
        K = None
        u = torch.tensor(rng.standard_normal(n) * 0.1 - np.log(n) + 2.0, dtype=torch.float32, device=dev)
        v = torch.tensor(rng.standard_normal(n) * 0.1, dtype=torch.float32, device=dev)
        U = torch.tensor(rng.standard_normal(n) * 0.01, dtype=torch.float64, device=dev)
        V = torch.tensor(rng.standard_normal(n) * 0.01, dtype=torch.float64, device=dev)
    Ad = nx.to_numpy_array(g, nodelist=range(n))
    Bd = nx.to_numpy_array(h, nodelist=range(n))
    return dict(n=n, ld=ld, A=A, B=B, Ad=Ad, Bd=Bd, P=P, C=C, K=K, u=u, v=v, U=U, V=V)


def _host(x):
    return None if x is None else x.cpu().numpy().astype(np.float64)


def _oracle_sums(s, reg):
    n = s["n"]
    P0, C0 = _host(s["P"])[:, :n], _host(s["C"])[:, :n]
    u0, v0 = _host(s["u"]), _host(s["v"])
    if s["K"] is not None:
        q = _host(s["K"])[:, :n] * v0[None, :] * u0[:, None]
        G = C0
    else:
        q = np.exp(C0 + u0[:, None] + v0[None, :])
        G = -reg * (C0 - _host(s["U"])[:, None] - _host(s["V"])[None, :])
    d = q - P0
    ADB = O.apb(s["Ad"], s["Bd"], d)
    sums = np.array([np.sum(G * d), np.sum(d * d), -2.0 * np.sum(d * ADB)])
    scale = np.array([np.sum(np.abs(G * d)), np.sum(d * d), 2.0 * np.sum(np.abs(d * ADB))])
    return P0, d, sums, scale


def _run_device(s, reg, lambda_eff):
    from cugal_b200 import _native as N
    n, ld = s["n"], s["ld"]
    dev = s["P"].device
    dirb = torch.zeros((n, ld), dtype=torch.float32, device=dev)
    W = torch.zeros((n, ld), dtype=torch.float32, device=dev)
    sums = torch.zeros(3, dtype=torch.float64, device=dev)
    alpha = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    gap = torch.zeros(1, dtype=torch.float64, device=dev)
    ws = torch.empty(N.workspace_size("fugal_gradient_workspace_size", n), dtype=torch.uint8, device=dev)
    stream = N.stream_handle()
    P = s["P"].clone()
    U = None if s["U"] is None else s["U"].clone()
    V = None if s["V"] is None else s["V"].clone()
    N.call("fugal_fw_direction", n, P.data_ptr(), ld, s["C"].data_ptr(), ld, N.ptr(s["K"]),
           ld if s["K"] is not None else 0, s["u"].data_ptr(), s["v"].data_ptr(), N.ptr(U), N.ptr(V), reg,
           dirb.data_ptr(), ld, sums.data_ptr(), 0 if U is None else 1, stream)
    N.call("fugal_fw_gradient", n, s["A"].row_pointers.data_ptr(), s["A"].col_indices.data_ptr(),
           s["B"].row_pointers.data_ptr(), s["B"].col_indices.data_ptr(), dirb.data_ptr(), ld, None, None, None, 0,
           0.0, 1.0, 1.0, None, None, W.data_ptr(), ld, ws.data_ptr(), ws.numel(), stream)
    N.call("fugal_fw_line_search_update", n, P.data_ptr(), ld, dirb.data_ptr(), ld, W.data_ptr(), ld,
           float(lambda_eff), sums.data_ptr(), alpha.data_ptr(), gap.data_ptr(), stream)
    torch.cuda.synchronize()
    return dict(P=P[:, :n].cpu().numpy().astype(np.float64), d=dirb[:, :n].cpu().numpy().astype(np.float64),
                sums=sums.cpu().numpy(), alpha=float(alpha.item()), gap=float(gap.item()), U=_host(U), V=_host(V))


@pytest.mark.parametrize("standard", [False, True])
@pytest.mark.parametrize("regime", ["interior", "clipped", "concave", "tiny", "ascent"])
def test_line_search_step_matches_oracle(standard, regime):
    s = _inputs(301, 5, standard)
    reg = 0.01
    if regime == "ascent":
        # flip the sign of G (the log form reads it as -reg (L - U - V), the scaling form as C)
        if standard:
            s["C"] = -s["C"]
        else:
            reg = -reg
    P0, d, sums, scale = _oracle_sums(s, reg)
    g, dd, dW = sums
    assert (g > 0) if regime == "ascent" else (g < 0), "inputs are built so that q - P descends"
    # lambda_eff that puts Q = dW/2 - lambda dd where each branch of the rule needs it
    Q_target = {"interior": -g, "clipped": -g / 4.0, "concave": -abs(g), "tiny": -g * 1e6,
                "ascent": -g / 2.0}[regime]
    expect = {"interior": 0.5, "clipped": 1.0, "concave": 1.0, "tiny": 5e-7, "ascent": 0.0}[regime]
    lam = (0.5 * dW - Q_target) / dd
    out = _run_device(s, reg, lam)
    np.testing.assert_allclose(out["sums"], sums, rtol=0, atol=1e-5 * scale.max())
    np.testing.assert_allclose(out["d"], d, rtol=1e-5, atol=1e-7)
    Qd = 0.5 * out["sums"][2] - lam * out["sums"][1]
    assert out["alpha"] == pytest.approx(O.line_search_alpha(out["sums"][0], Qd), rel=1e-12, abs=1e-15)
    a_ref = O.line_search_alpha(g, 0.5 * dW - lam * dd)
    assert a_ref == pytest.approx(expect, rel=1e-9, abs=1e-15)
    assert out["alpha"] == pytest.approx(a_ref, rel=1e-4, abs=1e-15)
    assert out["gap"] == out["sums"][0]
    np.testing.assert_allclose(out["P"], P0 + out["alpha"] * out["d"], rtol=0, atol=1e-6)
    if not standard:
        np.testing.assert_allclose(out["U"], _host(s["U"]) + _host(s["u"]), rtol=0, atol=1e-12)
        np.testing.assert_allclose(out["V"], _host(s["V"]) + _host(s["v"]), rtol=0, atol=1e-12)


def _pair(n, seed):
    from cugal_b200.synthetic import noisy_permuted_copy
    g = nx.newman_watts_strogatz_graph(n, 6, 0.1, seed=seed)
    h, perm = noisy_permuted_copy(g, np.random.default_rng(seed), 3, 3)
    return g, h, perm


@pytest.mark.parametrize("method,reg", [("LOG", 0.05), ("LOG", 0.5), ("STANDARD", 0.5)])
def test_alignment_with_line_search_matches_oracle(method, reg):
    from cugal_b200 import Config, HungarianMethod, Profile, SinkhornMethod, cugal
    n = 60
    g, h, perm = _pair(n, 7)
    params = dict(sinkhorn_regularization=reg, sinkhorn_iterations=300, sinkhorn_threshold=1e-6,
                  sinkhorn_eval_freq=10, mu=1.0, iter_count=3, frank_wolfe_iter_count=10)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod[method],
                 use_sparse_adjacency=True, hungarian_method=HungarianMethod.SCIPY, line_search=True, **params)
    prof = Profile()
    P, mapping = cugal(nx.Graph(g), nx.Graph(h), cfg, prof)
    trace = O.FWTrace()
    Pr, mref, _ = O.cugal(nx.Graph(g), nx.Graph(h),
                          O.OracleParams(sinkhorn_method=method, use_sparse_adjacency=True, hungarian_method="SCIPY",
                                         line_search=True, **params), features="cuda", trace=trace)
    steps = prof.frank_wolfe_steps
    assert len(steps) == len(trace.alphas) == 30
    assert all(0.0 <= a <= 1.0 for a in steps)
    # where the direction carries weight the steps agree; a vanishing direction moves P by nothing either way
    big = np.asarray(trace.gaps) > 1e-6 * max(trace.gaps)
    np.testing.assert_allclose(np.asarray(steps)[big], np.asarray(trace.alphas)[big], atol=1e-3)
    assert [m[1] for m in mapping] == [m[1] for m in mref]
    np.testing.assert_allclose(P, Pr, atol=2e-3)
