"""The kept structural term A P B (cugal_b200/structural.py) on the GPU.

* Kernel level, exact: with plans of ones and zeros and steps of 1/2, every value
  involved is a short dyadic fraction, so the recurrence (update that records the
  plan, scatter of a A q B) must give the same integers as a dense refresh of the
  updated P, and the gradient read from it must equal the SpMM gradient bit for bit.
* Flags: a plan row with more entries than the slots, or with a row sum above the
  bound, flags the step, and the next gradient recomputes Mq from P.
* Engine level: an alignment with the kept term against one with the SpMM
  gradient every step (FUGAL_GRAD_RECURRENCE=0), and rerun determinism."""

import networkx as nx
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _graphs(n, seed):
    from cugal_b200.synthetic import noisy_permuted_copy
    g = nx.gnp_random_graph(n, 0.05, seed=seed)
    h, _ = noisy_permuted_copy(g, np.random.default_rng(seed), 3, 3)
    return g, h


def _setup(n=256, seed=0):
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.sinkhorn import padded_ld
    from cugal_b200.structural import StructuralTerm
    from cugal_b200 import _native as N
    g, h = _graphs(n, seed)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    ld = padded_ld(n)
    ws = torch.empty(N.workspace_size("fugal_gradient_workspace_size", n), dtype=torch.uint8, device="cuda")
    st = StructuralTerm(A, B, n, ld, torch.device("cuda"), ws)
    P = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    P[:, :n] = 1.0 / n
    return A, B, ld, ws, st, P


def _refresh(st, P, bits):
    from cugal_b200 import _native as N
    Mq = torch.empty_like(st.Mq)
    flags = torch.zeros(2, dtype=torch.int32, device="cuda")
    N.call("fugal_structural_refresh", st.n, st.A.row_pointers.data_ptr(), st.A.col_indices.data_ptr(),
           st.B.row_pointers.data_ptr(), st.B.col_indices.data_ptr(), P.data_ptr(), st.ld, Mq.data_ptr(), st.ld,
           bits, st.workspace.data_ptr(), st.workspace.numel(), flags.data_ptr(), N.stream_handle("cuda"))
    assert flags.tolist() == [0, 0]
    return Mq


def _plan_cost(n, ld, rng, extra_rows=()):
    """cost32 whose plan q = exp(L) is 1 on a permutation (and on a second column
    of each row in extra_rows) and exactly 0 (expf(-200)) elsewhere."""
    L = torch.full((n, ld), -200.0, dtype=torch.float32)
    perm = rng.permutation(n)
    L[torch.arange(n), torch.as_tensor(perm)] = 0.0
    for r in extra_rows:
        L[r, (perm[r] + 1 + r) % n] = 0.0
    return L.cuda()


def test_recurrence_is_exact_on_dyadic_steps():
    from cugal_b200 import _native as N
    n = 256
    A, B, ld, ws, st, P = _setup(n)
    rng = np.random.default_rng(7)
    assert st.prepare(P)                       # refresh at P = 1/n
    bits = st.fixed.bits
    z32 = torch.zeros(ld, dtype=torch.float32, device="cuda")
    z64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    gap = torch.zeros(1, dtype=torch.float64, device="cuda")
    for t in range(1, 8):
        L = _plan_cost(n, ld, rng, extra_rows=range(0, n - 1, 17))
        st.collect_update(P, L, z32, z32, z64, z64, 0.5, 1e-3, gap)
        torch.cuda.synchronize()
        assert st.flags.tolist() == [0, 0]
        counts = st.counts.cpu().numpy()
        assert counts.sum() == n + len(range(0, n - 1, 17)) and counts.max() == 2
        assert st.fixed.scale == 0.5 ** t
        dense = _refresh(st, P, bits)
        assert torch.equal(st.Mq[:, :n], dense[:, :n] * (2 ** t)), t

    # the gradient read from Mq equals the SpMM gradient bit for bit (features,
    # lambda term, absorbed FP64 frame, column partials); with the shift folded in,
    # Mq comes back divided by 2^7, i.e. equal to the dense refresh
    fs = torch.tensor(rng.random((n, 4)) * 3, dtype=torch.float32, device="cuda")
    ft = torch.tensor(rng.random((n, 4)) * 3, dtype=torch.float32, device="cuda")
    U = torch.tensor(rng.standard_normal(n) * 1e3, device="cuda")
    V = torch.tensor(rng.standard_normal(n) * 1e3, device="cuda")
    chunks = (n + 127) // 128
    out_d = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    out_s = torch.zeros_like(out_d)
    part_d = torch.zeros((chunks, 2 * ld), dtype=torch.float32, device="cuda")
    part_s = torch.zeros_like(part_d)
    stream = N.stream_handle("cuda")
    N.call("fugal_fw_gradient_column_stats", n, A.row_pointers.data_ptr(), A.col_indices.data_ptr(),
           B.row_pointers.data_ptr(), B.col_indices.data_ptr(), P.data_ptr(), ld, fs.data_ptr(), ft.data_ptr(), None,
           0, 3.0, 1.0, -1e3, U.data_ptr(), V.data_ptr(), out_d.data_ptr(), ld, ws.data_ptr(), ws.numel(),
           part_d.data_ptr(), ld, stream)
    k = st.fixed.shift()
    assert k == 7
    N.call("fugal_fw_gradient_structural", n, st.Mq.data_ptr(), ld, st.fixed.m_scale(), k, P.data_ptr(), ld,
           fs.data_ptr(), ft.data_ptr(), None, 0, 3.0, 1.0, -1e3, U.data_ptr(), V.data_ptr(), out_s.data_ptr(), ld,
           part_s.data_ptr(), ld, stream)
    st.fixed.shifted(k)
    torch.cuda.synchronize()
    assert torch.equal(out_s[:, :n], out_d[:, :n])
    pd = part_d.view(chunks, ld, 2)[:, :n]
    ps = part_s.view(chunks, ld, 2)[:, :n]
    assert torch.equal(ps[..., 0], pd[..., 0])
    torch.testing.assert_close(ps[..., 1], pd[..., 1], rtol=2e-5, atol=0)
    assert torch.equal(st.Mq[:, :n], _refresh(st, P, bits)[:, :n])
    assert st.fixed.scale == 1.0


@pytest.mark.parametrize("case", ["too_many_entries", "row_sum"])
def test_flagged_plan_row_forces_a_refresh(case):
    from cugal_b200 import structural as S
    n = 256
    A, B, ld, ws, st, P = _setup(n, seed=3)
    assert st.prepare(P)
    L = torch.full((n, ld), -200.0, dtype=torch.float32, device="cuda")
    L[torch.arange(n), torch.arange(n)] = 0.0
    if case == "too_many_entries":
        L[5, :S.SLOTS + 3] = -1.0                 # 35 nonzero entries in row 5
    else:
        L[9, :10] = 2.0                           # ten entries of e^2: row sum 73.9 > 32
    z32 = torch.zeros(ld, dtype=torch.float32, device="cuda")
    z64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    gap = torch.zeros(1, dtype=torch.float64, device="cuda")
    st.collect_update(P, L, z32, z32, z64, z64, 0.5, 1e-3, gap)
    torch.cuda.synchronize()
    assert st.flags.tolist()[0] == 1
    if case == "too_many_entries":
        assert st.counts[5].item() == S.SLOTS + 3
    # the next gradient's prepare sees the flag and recomputes from the new P
    assert st.prepare(P)
    assert st.refreshes == 2 and st.fixed.scale == 1.0
    assert torch.equal(st.Mq[:, :n], _refresh(st, P, st.fixed.bits)[:, :n])


def _run(monkeypatch, recurrence: bool, n=1500, steps=(4, 6), seed=11, check=None):
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.feature_extraction import Features
    from cugal_b200.pred import FrankWolfeEngine
    from cugal_b200.synthetic import noisy_permuted_copy
    monkeypatch.setenv("FUGAL_GRAD_RECURRENCE", "1" if recurrence else "0")
    g = nx.newman_watts_strogatz_graph(n, 8, 0.1, seed=seed)
    h, perm = noisy_permuted_copy(g, np.random.default_rng(seed), 10, 10)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 sinkhorn_regularization=1e-3, sinkhorn_iterations=300, sinkhorn_threshold=1e-4, sinkhorn_eval_freq=10,
                 mu=1.0, iter_count=steps[0], frank_wolfe_iter_count=steps[1], use_sparse_adjacency=True,
                 stream_dtype=torch.bfloat16)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    eng = FrankWolfeEngine(A, B, Features.create(A, B, cfg), cfg, max_solves=steps[0] * steps[1])
    for lam in range(cfg.iter_count):
        for it in range(1, cfg.frank_wolfe_iter_count + 1):
            eng.gradient(lam)
            if check is not None:
                check(eng, lam)
            eng.solve()
            eng.update(2.0 / (2.0 + it), lam)
    torch.cuda.synchronize()
    return eng, perm


def test_kept_term_matches_spmm_gradient_on_the_same_p(monkeypatch):
    """At every step of an alignment, the kept A P B and the gradient read from it
    against the two-SpMM gradient of the same P and duals.  They differ by FP32
    rounding only: the kept term follows P' = (1 - a) P + a q exactly (to 2^-F),
    while P itself is rounded to FP32 at every update and the SpMM sums in FP32."""
    reg = 1e-3
    worst = {"m_rel": 0.0, "cost": 0.0}
    seen = []

    def check(eng, lam):
        st = eng.structural
        n = eng.n
        dense = eng.gradient(lam, out_scale=-1.0 / reg, out=torch.empty_like(eng.cost32))
        scale = max(1.0, dense[:, :n].abs().max().item())
        diff = (eng.cost32[:, :n] - dense[:, :n]).abs().max().item()
        M_rec = st.Mq[:, :n].double() * (st.fixed.scale * 2.0 ** -st.fixed.bits)
        M_den = _refresh(st, eng.P_buf, st.fixed.bits)[:, :n].double() * 2.0 ** -st.fixed.bits
        m_rel = ((M_rec - M_den).abs().max() / M_den.abs().max()).item()
        worst["m_rel"] = max(worst["m_rel"], m_rel)
        worst["cost"] = max(worst["cost"], diff)
        seen.append((st.refreshes, st.scatters, m_rel, diff, scale))
        # P drifts from the exact recurrence by at most one FP32 rounding per update,
        # and the SpMM pair rounds sums of up to deg_A + deg_B terms (NWS k = 8, p = 0.1)
        assert m_rel <= 2.0 ** -24 * (len(seen) + 64), seen[-1]
        # in nats: 2/reg times the absolute error of A P B, plus the FP64 frame's rounding
        assert diff <= 2.0 / reg * m_rel * M_den.abs().max().item() * 1.5 + 1e-6 * scale + 1e-2, seen[-1]

    eng, perm = _run(monkeypatch, True, check=check)
    st = eng.structural
    steps = len(seen)
    print("kept term per step (refreshes, scatters, rel err of A P B, max |d cost| nats, |cost|):", seen)
    print("worst:", worst)
    # the plan is spread over many columns only in the first steps
    assert st.scatters >= steps // 2 and st.refreshes <= steps // 2, (st.scatters, st.refreshes)
    eng_d, _ = _run(monkeypatch, False)
    assert eng_d.structural is None
    acc = lambda P: float(np.mean(P.argmax(axis=1) == perm))
    assert acc(eng.P.cpu().numpy()) == pytest.approx(acc(eng_d.P.cpu().numpy()), abs=5e-3)


def test_kept_term_reruns_are_bit_identical(monkeypatch):
    eng1, _ = _run(monkeypatch, True, n=1200, steps=(2, 5), seed=4)
    eng2, _ = _run(monkeypatch, True, n=1200, steps=(2, 5), seed=4)
    assert eng1.structural.scatters > 0
    assert torch.equal(eng1.P, eng2.P)
    assert torch.equal(eng1.structural.Mq, eng2.structural.Mq)


@pytest.mark.parametrize("n", [250, 384])
@pytest.mark.parametrize("distance", ["features", "stored", "none"])
@pytest.mark.parametrize("partials", [True, False])
def test_structural_gradient_equals_spmm_gradient(n, distance, partials):
    """Every form of the kept-term gradient against the SpMM gradient of the same
    dyadic P, bit for bit: the distance from features, from a stored matrix, or
    none; with and without column partials; n not a multiple of the tiles (250)."""
    from cugal_b200 import _native as N
    A, B, ld, ws, st, P = _setup(n, seed=n)
    P[:, :n] = 1.0 / 256
    rng = np.random.default_rng(n)
    assert st.prepare(P)
    z32 = torch.zeros(ld, dtype=torch.float32, device="cuda")
    z64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    gap = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(3):
        st.collect_update(P, _plan_cost(n, ld, rng, extra_rows=range(1, n - 1, 13)), z32, z32, z64, z64, 0.5, 1e-3,
                          gap)
    torch.cuda.synchronize()
    assert st.flags.tolist() == [0, 0]
    fs = ft = D = None
    if distance == "features":
        fs = torch.tensor(rng.random((n, 4)) * 3, dtype=torch.float32, device="cuda")
        ft = torch.tensor(rng.random((n, 4)) * 3, dtype=torch.float32, device="cuda")
    elif distance == "stored":
        D = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
        D[:, :n] = torch.tensor(rng.random((n, n)) * 5, dtype=torch.float32, device="cuda")
    U = torch.tensor(rng.standard_normal(n) * 1e3, device="cuda")
    V = torch.tensor(rng.standard_normal(n) * 1e3, device="cuda")
    chunks = (n + 127) // 128
    out_d = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    out_s = torch.zeros_like(out_d)
    part_d = torch.zeros((chunks, 2 * ld), dtype=torch.float32, device="cuda")
    part_s = torch.zeros_like(part_d)
    stream = N.stream_handle("cuda")
    dist_args = (N.ptr(fs), N.ptr(ft), N.ptr(D), ld if D is not None else 0)
    common = (*dist_args, 3.0, 1.0, -1e3, U.data_ptr(), V.data_ptr())
    graphs = (A.row_pointers.data_ptr(), A.col_indices.data_ptr(), B.row_pointers.data_ptr(),
              B.col_indices.data_ptr(), P.data_ptr(), ld)
    if partials:
        N.call("fugal_fw_gradient_column_stats", n, *graphs, *common, out_d.data_ptr(), ld, ws.data_ptr(),
               ws.numel(), part_d.data_ptr(), ld, stream)
    else:
        N.call("fugal_fw_gradient", n, *graphs, *common, out_d.data_ptr(), ld, ws.data_ptr(), ws.numel(), stream)
    N.call("fugal_fw_gradient_structural", n, st.Mq.data_ptr(), ld, st.fixed.m_scale(), 0, P.data_ptr(), ld,
           *common, out_s.data_ptr(), ld, part_s.data_ptr() if partials else None, ld, stream)
    torch.cuda.synchronize()
    assert torch.equal(out_s[:, :n], out_d[:, :n])
    if partials:
        pd = part_d.view(chunks, ld, 2)[:, :n]
        ps = part_s.view(chunks, ld, 2)[:, :n]
        assert torch.equal(ps[..., 0], pd[..., 0])
        torch.testing.assert_close(ps[..., 1], pd[..., 1], rtol=2e-5, atol=0)
