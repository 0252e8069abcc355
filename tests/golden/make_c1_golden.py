"""Golden alignment of the 1000-node Newman-Watts-Strogatz workload, produced by
the reference's own CPU implementation in FP64.

    python tests/golden/make_c1_golden.py     # CUGAL_REFERENCE: the cuGAL checkout (as make_golden.py)

Workload (``cugal_b200.synthetic.make_pair("nws1000")``): source
``newman_watts_strogatz_graph(1000, 10, 0.1, seed=0)``, target = the source
relabelled by ``default_rng(0).permutation(1000)`` with 1% of the edges removed
and as many non-edges added.  Config: mu 1, 15 lambda steps x 10 Frank-Wolfe
steps, log-domain Sinkhorn (reg 1e-3, at most 500 sweeps, marginal tolerance
1e-4 checked every 10 sweeps), SCIPY rounding, ``device='cpu'``,
``dtype=torch.float64``.

Two variants are recorded:

* ``dense`` -- the reference's CPU path as it ships (``use_sparse_adjacency=False``,
  ``dense_gradient``, whose lambda term is doubled: ``cugal/pred.py:45-50``);
* ``sparse`` -- the same run with the lambda term counted once, the semantics of
  the reference's sparse GPU path (``cugal/pred.py:54-74``); the dense gradient
  is swapped for one without the doubled term, because the reference's sparse
  product has no usable CPU branch (``cugal/adjacency.py:128-156`` loops over
  n^2 Python-level sums).

Both run with the reference's convergence check made non-mutating (the form it
leaves unreachable at ``cugal/sinkhorn.py:76``); as shipped, the check rescales
K in place and never passes, so every solve would run the full 500 sweeps.

Per variant the fixture holds: the mapping, node accuracy against the planted
permutation, per-solve Sinkhorn iteration counts and recorded errors, the
objective values at the returned plan, and the plan itself as the entries
>= 1e-6 (row, column, value), which carry all but a negligible part of its
mass (the rest is recorded as ``tail_max`` / ``tail_mass``).  The plan of the
dense variant takes about 4 minutes on 8 cores.
"""

from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import networkx as nx
import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from make_golden import import_reference, patched_marginal_error_log  # noqa: E402

ENTRY_MIN = 1e-6


def objectives(P: np.ndarray, src: nx.Graph, tgt: nx.Graph, D: np.ndarray, lam: float) -> dict:
    """FP64 objective terms at plan P: the structural term <P, A P B>, the feature
    term <D, P> and the concave term <P, 1 - P> (FUGAL's objective is
    -<P, A P B> + <D, P> + lam <P, 1 - P>)."""
    n = P.shape[0]
    A = nx.to_scipy_sparse_array(src, nodelist=range(n), dtype=np.float64, format="csr")
    B = nx.to_scipy_sparse_array(tgt, nodelist=range(n), dtype=np.float64, format="csr")
    AP = A @ P
    APB = (B.T @ AP.T).T
    structural = float(np.sum(P * APB))
    feature = float(np.sum(D * P))
    concave = float(np.sum(P * (1.0 - P)))
    return {"structural": structural, "feature": feature, "concave": concave,
            "objective": -structural + feature + lam * concave}


def main():
    torch.set_num_threads(os.cpu_count() or 1)
    cugal = import_reference()
    import cugal.pred as pred
    from cugal.config import Config, HungarianMethod, SinkhornMethod
    from cugal.feature_extraction import Features
    from cugal.profile import Profile
    from cugal.sinkhorn import SinkhornState
    from cugal_b200.synthetic import make_pair

    SinkhornState.marginal_error_log = patched_marginal_error_log
    original_dense = pred.dense_gradient

    def dense_gradient_lambda_once(A, B, P, features, iteration):
        gradient = -A.T @ P @ B - A @ P @ B.T
        gradient = pred.add_feature_distance(gradient, features)
        gradient += iteration - iteration * 2 * P
        return gradient

    src, tgt, perm, w = make_pair("nws1000")
    n = src.number_of_nodes()
    out = {"src_edges": np.array(sorted(src.edges()), dtype=np.int32),
           "tgt_edges": np.array(sorted(tgt.edges()), dtype=np.int32), "perm": perm.astype(np.int32)}
    for variant in ["dense", "sparse"]:
        pred.dense_gradient = original_dense if variant == "dense" else dense_gradient_lambda_once
        config = Config(device="cpu", dtype=torch.float64, sinkhorn_method=SinkhornMethod.LOG,
                        sinkhorn_regularization=1e-3, sinkhorn_iterations=500, sinkhorn_threshold=1e-4,
                        sinkhorn_eval_freq=10, mu=1.0, iter_count=15, frank_wolfe_iter_count=10,
                        use_sparse_adjacency=False, hungarian_method=HungarianMethod.SCIPY)
        profile = Profile()
        t0 = time.perf_counter()
        P, mapping = pred.cugal(nx.Graph(src), nx.Graph(tgt), config, profile)
        secs = time.perf_counter() - t0
        cols = np.array([m[1] for m in mapping], dtype=np.int32)
        feats = Features.create(nx.Graph(src), nx.Graph(tgt), config)
        D = feats.distance_matrix().numpy()
        lam = (config.iter_count - 1) * (2.0 if variant == "dense" else 1.0)
        obj = objectives(P, src, tgt, D, lam)
        rows, colsP = np.nonzero(P >= ENTRY_MIN)
        tail = np.where(P >= ENTRY_MIN, 0.0, P)
        pre = f"{variant}_"
        out[pre + "cols"] = cols
        out[pre + "accuracy"] = np.float64(np.mean(cols == perm))
        out[pre + "sk_iters"] = np.array([p.iteration_count for p in profile.sinkhorn_profiles], dtype=np.int32)
        out[pre + "sk_final_error"] = np.array([p.errors[-1] if p.errors else np.nan
                                                for p in profile.sinkhorn_profiles], dtype=np.float64)
        out[pre + "entry_rows"] = rows.astype(np.int32)
        out[pre + "entry_cols"] = colsP.astype(np.int32)
        out[pre + "entry_vals"] = P[rows, colsP].astype(np.float64)
        out[pre + "tail_max"] = np.float64(tail.max())
        out[pre + "tail_mass"] = np.float64(tail.sum())
        out[pre + "row_sums"] = P.sum(axis=1)
        out[pre + "col_sums"] = P.sum(axis=0)
        out[pre + "lambda_final"] = np.float64(lam)
        for k, v in obj.items():
            out[pre + k] = np.float64(v)
        out[pre + "seconds"] = np.float64(secs)
        out[pre + "threads"] = np.int64(torch.get_num_threads())
        print(f"{variant}: {secs:.1f} s, accuracy {out[pre + 'accuracy']:.4f}, objective {obj['objective']:.6f}, "
              f"mean sweeps {out[pre + 'sk_iters'].mean():.2f}, {rows.size} entries >= {ENTRY_MIN:g}", flush=True)
    pred.dense_gradient = original_dense
    np.savez_compressed(HERE / "reference_nws1000.npz", **out)
    print("wrote", HERE / "reference_nws1000.npz")


if __name__ == "__main__":
    main()
