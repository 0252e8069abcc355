"""GPU parity of the Frank-Wolfe step against the FP64 oracle: gradient, Sinkhorn
solve (FP32, BF16, FP16 streams; single CTA and cluster paths), update, the
reference-compatible kernels, and whole alignments.

Tolerances: FP32 kernels 1e-5 relative on gradients/updates; Sinkhorn duals
within 2e-4 (absolute, nats) of the FP64 iterates; BF16-stream plans within 1e-2
and FP16-stream plans within 2e-3 (absolute, entries of a row-stochastic plan)
after the FP32 polish sweep."""

import os

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu


def _pair(n, seed):
    from cugal_b200.synthetic import noisy_permuted_copy
    g = nx.newman_watts_strogatz_graph(n, 6, 0.1, seed=seed)
    h, perm = noisy_permuted_copy(g, np.random.default_rng(seed), 3, 3)
    return g, h, perm


@pytest.mark.parametrize("n,lam,lscale", [(64, 0, 1.0), (257, 3, 1.0), (1000, 2, 2.0)])
def test_gradient_matches_oracle(n, lam, lscale):
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.feature_extraction import Features
    from cugal_b200.pred import FrankWolfeEngine
    g, h, _ = _pair(n, n)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    rng = np.random.default_rng(1)
    fs = (rng.random((n, 4)) * 5).astype(np.float32)
    ft = (rng.random((n, 4)) * 5).astype(np.float32)
    P = (rng.random((n, n)) / n).astype(np.float32)
    feats = Features(torch.tensor(fs, device="cuda"), torch.tensor(ft, device="cuda"))
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 use_sparse_adjacency=lscale == 1.0, sinkhorn_regularization=1.0)
    eng = FrankWolfeEngine(A, B, feats, cfg)
    eng.P_buf[:, :n] = torch.tensor(P, device="cuda")
    out = torch.empty_like(eng.P_buf)
    G = eng.gradient(lam, out_scale=1.0, out=out, absorbed=False)[:, :n].cpu().numpy().astype(np.float64)
    Asp = O.csr_to_scipy(*O.csr_from_graph(g), n)
    Bsp = O.csr_to_scipy(*O.csr_from_graph(h), n)
    D = O.distance_matrix(fs, ft)
    ref = O.sparse_gradient(Asp, Bsp, P.astype(np.float64), D, lam * lscale)
    np.testing.assert_allclose(G, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())
    # stored distance matrix instead of features, absorbed output with FP64 duals
    eng2 = FrankWolfeEngine(A, B, torch.tensor(D, dtype=torch.float32, device="cuda"), cfg)
    eng2.P_buf[:, :n] = torch.tensor(P, device="cuda")
    eng2.U.copy_(torch.tensor(rng.standard_normal(n) * 1e3, device="cuda"))
    eng2.V.copy_(torch.tensor(rng.standard_normal(n) * 1e3, device="cuda"))
    L = eng2.gradient(lam, out_scale=-0.5)[:, :n].cpu().numpy().astype(np.float64)
    expect = -0.5 * ref + eng2.U.cpu().numpy()[:, None] + eng2.V.cpu().numpy()[None, :]
    np.testing.assert_allclose(L, expect, rtol=0, atol=2e-3 + 1e-6 * np.abs(expect).max())


@pytest.mark.parametrize("n", [64, 1000, 3000])
def test_gradient_column_stats(n):
    """fugal_fw_gradient_column_stats writes the same cost as fugal_fw_gradient, and
    its (max, sum) partials merge to the column log-sum-exp of that cost; a solve
    fed the partials matches one that reads the cost for its first column update."""
    import ctypes
    from cugal_b200 import _native as N
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.feature_extraction import Features
    from cugal_b200.pred import FrankWolfeEngine
    from cugal_b200.sinkhorn import read_record
    g, h, _ = _pair(n, n + 1)
    A, B = Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda")
    rng = np.random.default_rng(3)
    feats = Features(torch.tensor(rng.random((n, 4)) * 5, dtype=torch.float32, device="cuda"),
                     torch.tensor(rng.random((n, 4)) * 5, dtype=torch.float32, device="cuda"))
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, use_sparse_adjacency=True,
                 sinkhorn_regularization=0.05, sinkhorn_iterations=60, sinkhorn_threshold=1e-9, sinkhorn_eval_freq=10)
    eng = FrankWolfeEngine(A, B, feats, cfg, max_solves=2)
    eng.P_buf[:, :n] = torch.tensor(rng.random((n, n)) / n, dtype=torch.float32, device="cuda")
    eng.U.copy_(torch.tensor(rng.standard_normal(n) * 30, device="cuda"))
    eng.V.copy_(torch.tensor(rng.standard_normal(n) * 30, device="cuda"))
    plain = eng.gradient(2, out=torch.zeros_like(eng.P_buf))  # fugal_fw_gradient
    eng.gradient(2)                                            # the column-stats variant, into cost32
    assert eng.colpart_valid
    torch.cuda.synchronize()
    assert torch.equal(plain[:, :n], eng.cost32[:, :n])
    chunks = ctypes.c_int32()
    N.call("fugal_gradient_column_chunks", n, ctypes.byref(chunks))
    assert chunks.value == (n + 127) // 128 == eng.colpart.shape[0]
    part = eng.colpart.view(chunks.value, eng.ld, 2)[:, :n].double().cpu().numpy()
    M = part[..., 0].max(axis=0)
    lse = (M + np.log2(np.sum(part[..., 1] * np.exp2(part[..., 0] - M), axis=0))) * np.log(2)
    cost = eng.cost32[:, :n].double().cpu().numpy()
    cm = cost.max(axis=0)
    ref = cm + np.log(np.sum(np.exp(cost - cm), axis=0))
    np.testing.assert_allclose(lse, ref, rtol=0, atol=2e-5 * max(1.0, np.abs(ref).max()))
    # the solve with the partials against the solve that reads cost32 for them
    outs = []
    for use in (True, False):
        du = torch.zeros(n, dtype=torch.float32, device="cuda")
        dv = torch.zeros(n, dtype=torch.float32, device="cuda")
        rec = torch.empty(N.RECORD_BYTES, dtype=torch.uint8, device="cuda")
        eng.solver.solve(eng.cost32, du, dv, rec.data_ptr(), eng.colpart if use else None)
        outs.append((du.cpu().numpy(), dv.cpu().numpy(), read_record(rec.cpu())))
    (u1, v1, r1), (u2, v2, r2) = outs
    assert r1.iteration_count == r2.iteration_count
    shift = np.mean(u1 - u2)  # duals are defined up to u + c, v - c
    np.testing.assert_allclose(u1 - shift, u2, rtol=0, atol=1e-5 + 4e-6 * np.abs(u2).max())
    np.testing.assert_allclose(v1 + shift, v2, rtol=0, atol=1e-5 + 4e-6 * np.abs(v2).max())


def _solve_gpu(C, u0, v0, reg, max_iter, thr, freq, mstart=None, stream_dtype=None, polish=1, warmup=10,
               every=50):
    from cugal_b200 import _native as N
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.sinkhorn import SinkhornSolver, padded_ld, read_record
    n = C.shape[0]
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 sinkhorn_regularization=reg, sinkhorn_iterations=max_iter, sinkhorn_threshold=thr,
                 sinkhorn_eval_freq=freq, sinkhorn_momentum_start=mstart, stream_dtype=stream_dtype,
                 polish_sweeps=polish, fp32_warmup_sweeps=warmup, reabsorb_every=every)
    solver = SinkhornSolver(n, cfg, "cuda")
    K = -C / reg
    U, V = u0.astype(np.float64), v0.astype(np.float64)
    cost = torch.zeros((n, padded_ld(n)), dtype=torch.float32, device="cuda")
    cost[:, :n] = torch.tensor(K + U[:, None] + V[None, :], dtype=torch.float32, device="cuda")
    du = torch.empty(n, dtype=torch.float32, device="cuda")
    dv = torch.empty(n, dtype=torch.float32, device="cuda")
    rec = torch.empty(N.RECORD_BYTES, dtype=torch.uint8, device="cuda")
    solver.solve(cost, du, dv, rec.data_ptr())
    prof = read_record(rec.cpu())
    return U + du.cpu().numpy().astype(np.float64), V + dv.cpu().numpy().astype(np.float64), prof


def _plan(C, u, v, reg):
    return np.exp(-C / reg + u[:, None] + v[None, :])


# Launch shapes: n <= 2048 -> 128 threads x 16 columns, <= 4096 -> 128 x 32, else 256 x 32 with
# clusters of ceil(n / 8192) CTAs; FUGAL_SWEEP_SHAPE overrides.  Sizes are picked so that some
# CTA's slice has chunk-columns entirely past n (64, 500, 4104 and 8200 do).
@pytest.mark.parametrize("n,shape", [(64, None), (300, None), (500, None), (3000, None), (3000, "128,16"),
                                     (4104, "256,16"), (5000, None), (5000, "256,16")])
def test_sinkhorn_fp32_matches_oracle(n, shape, monkeypatch):
    if shape:
        monkeypatch.setenv("FUGAL_SWEEP_SHAPE", shape)
    rng = np.random.default_rng(n)
    C = rng.random((n, n)) * 4
    C = C.astype(np.float32).astype(np.float64)
    reg, freq = 0.05, 10
    max_iter = 30 if n >= 5000 else (60 if n >= 3000 else 200)
    # FP32 cannot push the summed column error below ~n * 1e-7; thresholds sit above that floor
    thr = 0.0 if n >= 3000 else 1e-3
    zero = np.zeros(n)
    ref = O.sinkhorn_log_solve(C, zero, zero, reg, max_iter, thr, freq)
    u, v, prof = _solve_gpu(C, zero, zero, reg, max_iter, thr, freq)
    assert abs(prof.iteration_count - ref.iteration_count) <= freq
    if ref.iteration_count < max_iter and min(abs(np.array(ref.errors) / thr - 1)) > 0.2:
        assert prof.iteration_count == ref.iteration_count
    k = min(len(prof.errors), len(ref.errors))
    np.testing.assert_allclose(prof.errors[:k], ref.errors[:k], rtol=2e-2, atol=5e-7 * n)
    # the two solutions share the same gauge (same iteration), compare duals and plans
    np.testing.assert_allclose(u, ref.u, atol=2e-4 * max(1.0, np.abs(ref.u).max() / 100))
    np.testing.assert_allclose(v, ref.v, atol=2e-4 * max(1.0, np.abs(ref.v).max() / 100))
    np.testing.assert_allclose(_plan(C, u, v, reg), _plan(C, ref.u, ref.v, reg), atol=1e-4)
    # warm-started second solve on a perturbed cost
    C2 = C + 0.3 * np.sin(np.arange(n * n)).reshape(n, n)
    C2 = C2.astype(np.float32).astype(np.float64)
    ref2 = O.sinkhorn_log_solve(C2, ref.u, ref.v, reg, max_iter, thr, freq)
    u2, v2, prof2 = _solve_gpu(C2, u, v, reg, max_iter, thr, freq)
    assert abs(prof2.iteration_count - ref2.iteration_count) <= freq
    np.testing.assert_allclose(_plan(C2, u2, v2, reg), _plan(C2, ref2.u, ref2.v, reg), atol=1e-4)


@pytest.mark.parametrize("n", [8200, 9000])
def test_sinkhorn_two_cta_cluster(n):
    # 256 threads x 32 columns per CTA, 2-CTA clusters; the second slice holds 8 / 808 columns
    rng = np.random.default_rng(9)
    C = (rng.random((n, n)) * 4).astype(np.float32).astype(np.float64)
    zero = np.zeros(n)
    ref = O.sinkhorn_log_solve(C, zero, zero, 0.05, 8, 0.0, 10)
    u, v, prof = _solve_gpu(C, zero, zero, 0.05, 8, 0.0, 10)
    assert prof.iteration_count == 8
    np.testing.assert_allclose(u, ref.u, atol=1e-4)
    np.testing.assert_allclose(_plan(C, u, v, 0.05), _plan(C, ref.u, ref.v, 0.05), atol=1e-4)


def test_sinkhorn_momentum_matches_oracle():
    n = 200
    rng = np.random.default_rng(5)
    C = (rng.random((n, n)) * 4).astype(np.float32).astype(np.float64)
    zero = np.zeros(n)
    # threshold above the FP32 floor (~n * 5e-8) so both stop on the same evaluation
    ref = O.sinkhorn_log_solve(C, zero, zero, 0.05, 300, 1e-4, 5, momentum_start=10)
    u, v, prof = _solve_gpu(C, zero, zero, 0.05, 300, 1e-4, 5, mstart=10)
    assert prof.iteration_count == ref.iteration_count
    np.testing.assert_allclose(prof.errors, ref.errors, rtol=2e-2, atol=5e-8 * n)
    np.testing.assert_allclose(_plan(C, u, v, 0.05), _plan(C, ref.u, ref.v, 0.05), atol=2e-4)


@pytest.mark.parametrize("kernel", ["rows", "cluster"])
@pytest.mark.parametrize("dtype,tol", [(torch.bfloat16, 1e-2), (torch.float16, 2e-3)])
@pytest.mark.parametrize("n", [300, 3000, 9000])
def test_sinkhorn_reduced_precision_stream(dtype, tol, n, kernel, monkeypatch):
    if kernel == "cluster":
        monkeypatch.setenv("FUGAL_ROW_SWEEP", "0")
    rng = np.random.default_rng(11)
    C = (rng.random((n, n)) * 4).astype(np.float32).astype(np.float64)
    zero = np.zeros(n)
    reg = 0.05
    iters, warmup, every = (12, 4, 4) if n > 8192 else (80, 5, 20)
    ref = O.sinkhorn_log_solve(C, zero, zero, reg, iters, 0.0, 10)
    u, v, prof = _solve_gpu(C, zero, zero, reg, iters, 0.0, 10, stream_dtype=dtype, polish=1, warmup=warmup,
                            every=every)
    assert prof.iteration_count == iters
    P, R = _plan(C, u, v, reg), _plan(C, ref.u, ref.v, reg)
    np.testing.assert_allclose(P, R, atol=tol)
    np.testing.assert_allclose(P.sum(axis=1), 1.0, atol=1e-4)  # rows exact after the FP32 polish sweep


def _solve_device(Ct, reg, max_iter, stream_dtype=None, polish=1, warmup=3, every=4, mstart=None):
    """Zero-start solve of the device cost Ct (n x n FP32, torch): (u, v) FP64 numpy."""
    from cugal_b200 import _native as N
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.sinkhorn import SinkhornSolver, padded_ld
    n = Ct.shape[0]
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 sinkhorn_regularization=reg, sinkhorn_iterations=max_iter, sinkhorn_threshold=0.0,
                 sinkhorn_eval_freq=10, stream_dtype=stream_dtype, polish_sweeps=polish, fp32_warmup_sweeps=warmup,
                 reabsorb_every=every, sinkhorn_momentum_start=mstart)
    solver = SinkhornSolver(n, cfg, "cuda")
    cost = torch.zeros((n, padded_ld(n)), dtype=torch.float32, device="cuda")
    cost[:, :n] = Ct / -reg
    du = torch.empty(n, dtype=torch.float32, device="cuda")
    dv = torch.empty(n, dtype=torch.float32, device="cuda")
    solver.solve(cost, du, dv, None)
    torch.cuda.synchronize()
    del solver, cost
    return du.cpu().numpy().astype(np.float64), dv.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("n,mstart", [(17000, None), (20000, None), (32768, None), (40000, None), (65536, None),
                                      (40000, 4)])
def test_row_sweep_matches_cluster_sweep_and_fp32(n, mstart, monkeypatch):
    """16-bit solves with the row-owned sweep (two row segments, padded columns;
    above 32768 columns a two-CTA cluster per row block, with momentum on the
    exact path in one case) against the cluster sweep and the FP32 stream on the
    same problem."""
    from cugal_b200 import _native as N
    plan = N.sinkhorn_plan(n, N.FUGAL_BF16)
    assert plan["threads"] == 512 and plan["cluster"] == (2 if n > 32768 else 1), plan
    g = torch.Generator(device="cuda").manual_seed(n)
    Ct = torch.rand((n, n), generator=g, device="cuda") * 4
    reg = 0.05
    kw = dict(mstart=mstart) if mstart else {}
    u_r, v_r = _solve_device(Ct, reg, 12, stream_dtype=torch.bfloat16, **kw)
    monkeypatch.setenv("FUGAL_ROW_SWEEP", "0")
    u_c, v_c = _solve_device(Ct, reg, 12, stream_dtype=torch.bfloat16, **kw)
    u_f, v_f = _solve_device(Ct, reg, 12, **kw)
    rows = np.random.default_rng(n).choice(n, 64, replace=False)
    Cs = Ct[torch.tensor(rows, device="cuda")].double().cpu().numpy()
    del Ct
    torch.cuda.empty_cache()
    P_r = np.exp(-Cs / reg + u_r[rows, None] + v_r[None, :])
    P_c = np.exp(-Cs / reg + u_c[rows, None] + v_c[None, :])
    P_f = np.exp(-Cs / reg + u_f[rows, None] + v_f[None, :])
    np.testing.assert_allclose(P_r, P_c, atol=1e-2)
    np.testing.assert_allclose(P_r, P_f, atol=1e-2)
    np.testing.assert_allclose(P_r.sum(axis=1), 1.0, atol=1e-3)


@pytest.mark.parametrize("warmup", [0, 1])
def test_reduced_precision_without_fp32_warmup(warmup):
    """The absorb sweep may be the first sweep of a solve (no FP32 warm-up)."""
    n = 3000
    rng = np.random.default_rng(5)
    C = (rng.random((n, n)) * 4).astype(np.float32).astype(np.float64)
    zero = np.zeros(n)
    reg = 0.05
    ref = O.sinkhorn_log_solve(C, zero, zero, reg, 40, 0.0, 10)
    u, v, prof = _solve_gpu(C, zero, zero, reg, 40, 0.0, 10, stream_dtype=torch.bfloat16, polish=1, warmup=warmup,
                            every=20)
    assert prof.iteration_count == 40
    np.testing.assert_allclose(_plan(C, u, v, reg), _plan(C, ref.u, ref.v, reg), atol=1e-2)


def test_row_sweep_momentum_matches_oracle():
    n = 3000
    rng = np.random.default_rng(21)
    C = (rng.random((n, n)) * 4).astype(np.float32).astype(np.float64)
    zero = np.zeros(n)
    reg = 0.05
    ref = O.sinkhorn_log_solve(C, zero, zero, reg, 60, 0.0, 10, 20)
    u, v, prof = _solve_gpu(C, zero, zero, reg, 60, 0.0, 10, mstart=20, stream_dtype=torch.bfloat16, polish=1,
                            warmup=3, every=20)
    assert prof.iteration_count == 60
    np.testing.assert_allclose(_plan(C, u, v, reg), _plan(C, ref.u, ref.v, reg), atol=1e-2)


def test_update_matches_oracle():
    from cugal_b200 import _native as N
    n = 301
    rng = np.random.default_rng(2)
    ld = 304
    P = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    P[:, :n] = torch.tensor(rng.random((n, n)) / n, dtype=torch.float32)
    L = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    L[:, :n] = torch.tensor(-rng.random((n, n)) * 6, dtype=torch.float32)
    u = torch.tensor(rng.standard_normal(n) * 0.1, dtype=torch.float32, device="cuda")
    v = torch.tensor(rng.standard_normal(n) * 0.1, dtype=torch.float32, device="cuda")
    U = torch.tensor(rng.standard_normal(n) * 100, dtype=torch.float64, device="cuda")
    V = torch.tensor(rng.standard_normal(n) * 100, dtype=torch.float64, device="cuda")
    P0, L0, U0, V0 = P.cpu().numpy()[:, :n].astype(np.float64), L.cpu().numpy()[:, :n].astype(np.float64), \
        U.cpu().numpy(), V.cpu().numpy()
    u0, v0 = u.cpu().numpy().astype(np.float64), v.cpu().numpy().astype(np.float64)
    gap = torch.zeros(1, dtype=torch.float64, device="cuda")
    reg, alpha = 0.01, 0.4
    N.call("fugal_fw_update", n, P.data_ptr(), ld, L.data_ptr(), ld, u.data_ptr(), v.data_ptr(), U.data_ptr(),
           V.data_ptr(), alpha, reg, gap.data_ptr(), 1, N.stream_handle())
    q = np.exp(L0 + u0[:, None] + v0[None, :])
    G = -reg * (L0 - U0[:, None] - V0[None, :])
    Pr = P0.copy()
    diff = O.update_quasi_permutation(Pr, L0, u0, v0, alpha)
    np.testing.assert_allclose(P.cpu().numpy()[:, :n], Pr, rtol=2e-6, atol=1e-9)
    np.testing.assert_allclose(gap.item(), np.sum((q - P0) * G), rtol=1e-5)
    np.testing.assert_allclose(O.duality_gap(G, diff, alpha), abs(gap.item()), rtol=1e-5)
    np.testing.assert_allclose(U.cpu().numpy(), U0 + u0, rtol=0, atol=1e-12)
    np.testing.assert_allclose(V.cpu().numpy(), V0 + v0, rtol=0, atol=1e-12)


def test_reference_compatible_kernels():
    from cugal_b200 import cuda_kernels as ck
    n = 129
    rng = np.random.default_rng(4)
    K = torch.tensor(rng.standard_normal((n, n)) * 3, dtype=torch.float32, device="cuda")
    add = torch.tensor(rng.standard_normal(n), dtype=torch.float32, device="cuda")
    out = torch.tensor(rng.standard_normal(n), dtype=torch.float32, device="cuda")
    Kh, ah, oh = (t.cpu().numpy().astype(np.float64) for t in (K, add, out))
    for w in (1.0, 1.3):
        o = out.clone()
        ck.sinkhorn_log_step(K, add, o, w)
        np.testing.assert_allclose(o.cpu().numpy(), O.sinkhorn_log_step(Kh, ah, oh, w), rtol=1e-5, atol=1e-5)
    u = torch.tensor(rng.standard_normal(n) * 0.1, dtype=torch.float32, device="cuda")
    v = torch.tensor(rng.standard_normal(n) * 0.1 - 4.0, dtype=torch.float32, device="cuda")
    Q = np.exp(Kh + u.cpu().numpy()[:, None] + v.cpu().numpy()[None, :])
    assert np.isclose(ck.sinkhorn_log_marginal(K, u, v), np.sum(np.abs(Q.sum(1) - 1)), rtol=1e-5)
    G = torch.tensor(rng.standard_normal((n, n)), dtype=torch.float32, device="cuda")
    P = torch.rand((n, n), device="cuda")
    G2 = G.clone()
    ck.regularize(G2, P, 3)
    expect = G.cpu().numpy() + (np.float32(3) - np.float32(6) * P.cpu().numpy())
    np.testing.assert_allclose(G2.cpu().numpy(), expect, rtol=0, atol=1e-6)
    fs = torch.rand((n, 4), device="cuda") * 5
    ft = torch.rand((n, 4), device="cuda") * 5
    D = torch.zeros((n, n), device="cuda")
    ck.add_distance(fs, ft, D)
    np.testing.assert_allclose(D.cpu().numpy(), O.distance_matrix(fs.cpu().numpy(), ft.cpu().numpy()),
                               rtol=1e-6, atol=1e-6)
    P2 = P.clone()
    gap = ck.update_quasi_permutation_log(P2, K, u, v, 0.25, 0.01)
    Pr = P.cpu().numpy().astype(np.float64)
    diff = O.update_quasi_permutation(Pr, Kh, u.cpu().numpy(), v.cpu().numpy(), 0.25)
    np.testing.assert_allclose(P2.cpu().numpy(), Pr, rtol=1e-5, atol=1e-6)
    assert np.isclose(gap, O.duality_gap(-0.01 * Kh, diff, 0.25), rtol=1e-4)


@pytest.mark.parametrize("lap", ["SCIPY", "DOUBLE_GREEDY"])
def test_full_alignment_matches_oracle(lap):
    from cugal_b200 import Config, HungarianMethod, Profile, SinkhornMethod, cugal
    n = 60
    g, h, perm = _pair(n, 7)
    params = dict(sinkhorn_regularization=0.05, sinkhorn_iterations=200, sinkhorn_threshold=1e-5,
                  sinkhorn_eval_freq=10, mu=1.0, iter_count=3, frank_wolfe_iter_count=10)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 use_sparse_adjacency=True, hungarian_method=HungarianMethod[lap], **params)
    prof = Profile()
    P, mapping = cugal(nx.Graph(g), nx.Graph(h), cfg, prof)
    trace = O.FWTrace()
    Pr, mref, sp32 = O.cugal(nx.Graph(g), nx.Graph(h),
                             O.OracleParams(sinkhorn_method="LOG", use_sparse_adjacency=True, hungarian_method=lap,
                                            **params), features="cuda", trace=trace,
                             sparsity_eps=float(np.finfo(np.float32).eps))
    assert prof.frank_wolfe_iterations == trace.frank_wolfe_iterations == 30
    its = [p.iteration_count for p in prof.sinkhorn_profiles]
    assert len(its) == 30
    assert max(abs(a - b) for a, b in zip(its, trace.sinkhorn_iterations)) <= 10
    assert [m[1] for m in mapping] == [m[1] for m in mref]
    np.testing.assert_allclose(P, Pr, atol=2e-3)
    # the reference's GPU path counts entries <= FP32 epsilon (its P is FP32), before rounding
    assert abs(prof.sparsity - sp32) < 0.02
    from cugal_b200 import Phase
    assert set(prof.phase_times) == set(Phase)


@pytest.mark.parametrize("threshold", [1e30, "mid"])
def test_frank_wolfe_threshold_early_stop(threshold):
    """frank_wolfe_threshold (cugal/pred.py:144): the lambda step's inner loop ends
    at the first Frank-Wolfe step whose duality gap is below the threshold; the
    steps taken and the plan match the oracle's."""
    from cugal_b200 import Config, HungarianMethod, Profile, SinkhornMethod, cugal
    n = 60
    g, h, perm = _pair(n, 7)
    params = dict(sinkhorn_regularization=0.05, sinkhorn_iterations=200, sinkhorn_threshold=1e-5,
                  sinkhorn_eval_freq=10, mu=1.0, iter_count=3, frank_wolfe_iter_count=10)
    oracle_kw = dict(sinkhorn_method="LOG", use_sparse_adjacency=True, hungarian_method="DOUBLE_GREEDY", **params)
    if threshold == "mid":
        # a threshold between the gaps of the full run: some lambda steps stop early, others do not
        full = O.FWTrace()
        O.cugal(nx.Graph(g), nx.Graph(h), O.OracleParams(**oracle_kw), features="cuda", trace=full)
        gaps = np.sort(np.array(full.gaps))
        # the widest ratio between neighbouring gaps in the middle half, so that FP32
        # rounding of the gaps cannot move a decision
        lo, hi = len(gaps) // 4, 3 * len(gaps) // 4
        k = lo + int(np.argmax(gaps[lo + 1:hi + 1] / gaps[lo:hi]))
        threshold = float(np.sqrt(gaps[k] * gaps[k + 1]))
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, use_sparse_adjacency=True,
                 hungarian_method=HungarianMethod.DOUBLE_GREEDY, frank_wolfe_threshold=threshold, **params)
    prof = Profile()
    P, mapping = cugal(nx.Graph(g), nx.Graph(h), cfg, prof)
    trace = O.FWTrace()
    Pr, mref, _ = O.cugal(nx.Graph(g), nx.Graph(h), O.OracleParams(frank_wolfe_threshold=threshold, **oracle_kw),
                          features="cuda", trace=trace)
    assert prof.frank_wolfe_iterations == trace.frank_wolfe_iterations
    if threshold == 1e30:
        assert trace.frank_wolfe_iterations == params["iter_count"]  # one step per lambda
    else:
        assert params["iter_count"] < trace.frank_wolfe_iterations < 30
    assert [m[1] for m in mapping] == [m[1] for m in mref]
    np.testing.assert_allclose(P, Pr, atol=2e-3)
