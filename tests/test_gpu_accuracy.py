"""Whole-path accuracy against FP64 references at the benchmark configurations.

* nws1000 -- Newman-Watts-Strogatz n=1000 (k 10, p 0.1, seed 0, 1% edge noise),
  mu 1, 15 x 10 Frank-Wolfe steps, log Sinkhorn reg 1e-3 (<= 500 sweeps,
  tolerance 1e-4), SCIPY rounding: the reference's own CPU FP64 run
  (``tests/golden/reference_nws1000.npz``, made by
  ``tests/golden/make_c1_golden.py``) against this path with an FP32 and a BF16
  stream, for the dense path's semantics (doubled lambda term) and the sparse
  path's.
* er32768 -- Erdos-Renyi n=32768 (mean degree 16, seed 2, 2% noise), same
  schedule, DOUBLE_GREEDY rounding: the torch FP64 restatement
  (``oracle/fugal_torch64.py``) on the GPU, truncated to the first lambda block
  (P, objective and per-solve sweep counts) and over the full schedule (node
  accuracy).

Quantities (each printed): node accuracy against the planted permutation, the
FUGAL objective -<P, A P B> + <D, P> + lam <P, 1 - P> evaluated in FP64 at the
returned plan, max |P - P_64| and the Sinkhorn sweep counts.
"""

from pathlib import Path

import networkx as nx
import numpy as np
import pytest
import torch

from oracle import fugal_fp64 as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_nws1000.npz"


def objective_fp64(P: np.ndarray, src: nx.Graph, tgt: nx.Graph, D: np.ndarray, lam: float) -> float:
    n = P.shape[0]
    A = nx.to_scipy_sparse_array(src, nodelist=range(n), dtype=np.float64, format="csr")
    B = nx.to_scipy_sparse_array(tgt, nodelist=range(n), dtype=np.float64, format="csr")
    P = P.astype(np.float64)
    APB = (B.T @ (A @ P).T).T
    return float(-np.sum(P * APB) + np.sum(D * P) + lam * np.sum(P * (1.0 - P)))


def plan_error_vs_entries(P: np.ndarray, g, prefix: str) -> float:
    """max |P - P_64| where P_64 is given by its entries >= 1e-6 (and is below
    1e-6 elsewhere)."""
    r, c, v = g[prefix + "entry_rows"], g[prefix + "entry_cols"], g[prefix + "entry_vals"]
    err_stored = float(np.max(np.abs(P[r, c].astype(np.float64) - v)))
    mask = np.zeros(P.shape, dtype=bool)
    mask[r, c] = True
    rest = np.where(mask, 0.0, P.astype(np.float64))
    err_rest = max(0.0, float(rest.max()) - 1e-6) if rest.size else 0.0
    return max(err_stored, err_rest)


@pytest.mark.skipif(not GOLDEN.exists(), reason="golden fixture of the 1000-node workload not generated")
@pytest.mark.parametrize("variant", ["dense", "sparse"])
@pytest.mark.parametrize("stream", ["fp32", "bf16"])
def test_nws1000_against_reference_fp64(variant, stream):
    from cugal_b200 import Profile, cugal
    from cugal_b200.synthetic import config_for, make_pair
    g = np.load(GOLDEN)
    src, tgt, perm, w = make_pair("nws1000")
    assert np.array_equal(np.array(sorted(src.edges()), dtype=np.int32), g["src_edges"])
    assert np.array_equal(np.array(sorted(tgt.edges()), dtype=np.int32), g["tgt_edges"])
    sdt = {"fp32": None, "bf16": torch.bfloat16}[stream]
    config = config_for(w, device="cuda", stream_dtype=sdt, use_sparse_adjacency=variant == "sparse")
    prof = Profile()
    P, mapping = cugal(nx.Graph(src), nx.Graph(tgt), config, prof)
    pre = variant + "_"
    cols = np.array([m[1] for m in mapping])
    acc = float(np.mean(cols == perm))
    D = O.distance_matrix(O.features_nx_semantics(src), O.features_nx_semantics(tgt))
    obj = objective_fp64(P, src, tgt, D, float(g[pre + "lambda_final"]))
    obj_ref = float(g[pre + "objective"])
    perr = plan_error_vs_entries(P, g, pre)
    sweeps = np.array([p.iteration_count for p in prof.sinkhorn_profiles])
    same_map = float(np.mean(cols == g[pre + "cols"]))
    print(f"\n[nws1000 {variant} {stream}] accuracy {acc:.4f} (FP64 reference {float(g[pre + 'accuracy']):.4f}); "
          f"objective {obj:.6f} vs {obj_ref:.6f} (rel {abs(obj - obj_ref) / abs(obj_ref):.2e}); "
          f"max|P-P64| {perr:.3e}; same column {same_map:.4f}; mean sweeps {sweeps.mean():.2f} vs "
          f"{g[pre + 'sk_iters'].mean():.2f}")
    # The lambda schedule drives P to a vertex and the NWS graph has many near-ties, so
    # rounding-level differences (FP32 or BF16 against FP64, FP32 against FP64 features,
    # the kept A P B against two SpMMs per step) move individual rows to other vertices:
    # max|P - P64| is 1 at those rows.  Two FP64 computations of the sparse path differ
    # by 1.3 pt (the reference's 0.685 against the numpy FP64 restatement's 0.698,
    # tests/golden/fp64_spread_nws1000.py); accuracy is held to that spread plus 0.2 pt,
    # objective within 1.5e-2 relative.  The same two FP64 runs put 91% of rows on the
    # same column; this path has measured 84.9-95.2% over the four configurations, so at
    # least 80% of rows must land on the reference's column.
    tol = 0.015
    assert abs(acc - float(g[pre + "accuracy"])) <= tol
    assert abs(obj - obj_ref) <= 1.5e-2 * abs(obj_ref)
    assert same_map >= 0.80


def _er32768_pair():
    from cugal_b200.synthetic import make_pair
    return make_pair("er32768")


def _oracle_run(src, tgt, steps=None, trace=None):
    from oracle import fugal_torch64 as T
    A_csr, B_csr = O.csr_from_graph(src), O.csr_from_graph(tgt)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    P = T.find_quasi_permutation_matrix(A_csr, B_csr, F1, F2, reg=1e-3, iter_count=15, fw_iter_count=10,
                                        sinkhorn_iterations=500, threshold=1e-4, eval_freq=10, mu=1.0,
                                        device="cuda", block=1024, max_steps=steps, trace=trace)
    return P, (A_csr, B_csr, F1, F2)


def _ours_truncated(src, tgt, stream, steps):
    from cugal_b200 import Profile
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.feature_extraction import Features
    from cugal_b200.pred import find_quasi_permutation_matrix
    from cugal_b200.synthetic import WORKLOADS, config_for
    sdt = {"fp32": None, "bf16": torch.bfloat16}[stream]
    config = config_for(WORKLOADS["er32768"], device="cuda", stream_dtype=sdt, iter_count=1,
                        frank_wolfe_iter_count=steps)
    A = Adjacency.from_graph(src, "cuda")
    B = Adjacency.from_graph(tgt, "cuda")
    prof = Profile()
    P = find_quasi_permutation_matrix(A, B, Features.create(A, B, config), config, prof)
    prof.resolve()
    return P, [p.iteration_count for p in prof.sinkhorn_profiles]


def test_er32768_first_lambda_block_against_fp64():
    from oracle import fugal_torch64 as T
    steps = 10
    src, tgt, perm, _ = _er32768_pair()
    trace = T.Trace()
    P64, (A_csr, B_csr, F1, F2) = _oracle_run(src, tgt, steps=steps, trace=trace)
    n = P64.shape[0]
    A = T.csr_tensor(*A_csr, n, "cuda")
    B = T.csr_tensor(*B_csr, n, "cuda")
    f1 = torch.as_tensor(F1, device="cuda")
    f2 = torch.as_tensor(F2, device="cuda")
    obj64 = T.objective(A, B, P64, f1, f2, 0.0, 1024)["objective"]
    for stream in ("fp32", "bf16"):
        P, sweeps = _ours_truncated(src, tgt, stream, steps)
        err = 0.0
        for r0 in range(0, n, 2048):
            err = max(err, float((P[r0:r0 + 2048].double() - P64[r0:r0 + 2048]).abs().max().item()))
        obj = T.objective(A, B, P.double(), f1, f2, 0.0, 1024)["objective"]
        rel = abs(obj - obj64) / abs(obj64)
        print(f"\n[er32768 first {steps} FW steps, {stream}] max|P-P64| {err:.3e}; objective {obj:.6f} vs "
              f"{obj64:.6f} (rel {rel:.2e}); sweeps {sweeps} vs FP64 {trace.sinkhorn_iterations}; "
              f"FP64 final errors {['%.1e' % e for e in trace.sinkhorn_final_errors]}")
        del P
        # measured: FP32 max|P - P64| 4.8e-4, BF16 2.2e-2; objective 5e-5 relative for both;
        # BF16 runs the FP64 solve's iteration counts, FP32 caps one more early solve
        assert rel <= 2e-4
        assert err <= (2e-3 if stream == "fp32" else 5e-2)
        if stream == "bf16":
            assert sweeps == trace.sinkhorn_iterations
    del P64
    torch.cuda.empty_cache()


def test_er32768_full_schedule_node_accuracy_against_fp64():
    from oracle import fugal_torch64 as T
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.pred import align
    from cugal_b200.synthetic import WORKLOADS, config_for
    src, tgt, perm, _ = _er32768_pair()
    trace = T.Trace()
    P64, _ = _oracle_run(src, tgt, trace=trace)
    cols64 = T.double_greedy(P64)
    acc64 = float(np.mean(cols64 == perm))
    del P64
    torch.cuda.empty_cache()
    A = Adjacency.from_graph(src, "cuda")
    B = Adjacency.from_graph(tgt, "cuda")
    for stream in ("fp32", "bf16"):
        sdt = {"fp32": None, "bf16": torch.bfloat16}[stream]
        config = config_for(WORKLOADS["er32768"], device="cuda", stream_dtype=sdt)
        _, cols, _ = align(A, B, config)
        acc = float(np.mean(cols.cpu().numpy() == perm))
        print(f"\n[er32768 full schedule {stream}] node accuracy {acc:.4f} vs FP64 {acc64:.4f}; FP64 mean sweeps "
              f"{np.mean(trace.sinkhorn_iterations):.2f}, capped solves "
              f"{int(np.sum(np.array(trace.sinkhorn_iterations) >= 500))}")
        assert abs(acc - acc64) <= 0.005


def test_ba8192_full_schedule_against_fp64():
    """Barabasi-Albert n=8192 (m 5, seed 1, 5% noise), the plain FP32 drop-in
    path with SCIPY rounding, against the FP64 restatement over the full
    15 x 10 schedule (its plan rounded by scipy): node accuracy and objective."""
    import scipy.optimize
    from oracle import fugal_torch64 as T
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.pred import align
    from cugal_b200.synthetic import config_for, make_pair
    src, tgt, perm, w = make_pair("ba8192")
    A_csr, B_csr = O.csr_from_graph(src), O.csr_from_graph(tgt)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    trace = T.Trace()
    P64 = T.find_quasi_permutation_matrix(A_csr, B_csr, F1, F2, reg=1e-3, iter_count=15, fw_iter_count=10,
                                          sinkhorn_iterations=500, threshold=1e-4, eval_freq=10, mu=1.0,
                                          device="cuda", block=1024, trace=trace)
    n = P64.shape[0]
    A = T.csr_tensor(*A_csr, n, "cuda")
    B = T.csr_tensor(*B_csr, n, "cuda")
    f1, f2 = torch.as_tensor(F1, device="cuda"), torch.as_tensor(F2, device="cuda")
    obj64 = T.objective(A, B, P64, f1, f2, 14.0, 1024)["objective"]
    cols64 = scipy.optimize.linear_sum_assignment(P64.cpu().numpy(), maximize=True)[1]
    acc64 = float(np.mean(cols64 == perm))
    del P64
    torch.cuda.empty_cache()
    config = config_for(w, device="cuda")
    P, cols, _ = align(Adjacency.from_graph(src, "cuda"), Adjacency.from_graph(tgt, "cuda"), config)
    cols = cols.cpu().numpy() if isinstance(cols, torch.Tensor) else np.asarray(cols)
    acc = float(np.mean(cols == perm))
    obj = T.objective(A, B, P.double(), f1, f2, 14.0, 1024)["objective"]
    rel = abs(obj - obj64) / abs(obj64)
    print(f"\n[ba8192 full schedule fp32, SCIPY] node accuracy {acc:.4f} vs FP64 {acc64:.4f}; objective {obj:.4f} vs "
          f"{obj64:.4f} (rel {rel:.2e}); same column {float(np.mean(cols == cols64)):.4f}; FP64 mean iterations "
          f"{np.mean(trace.sinkhorn_iterations):.1f}, capped {int(np.sum(np.array(trace.sinkhorn_iterations) >= 500))}")
    assert abs(acc - acc64) <= 0.005
    assert rel <= 1e-2
