"""How far two FP64 computations of the same 1000-node alignment drift apart.

    python tests/golden/fp64_spread_nws1000.py      # CPU, about 10-13 minutes per run

Runs the numpy FP64 oracle (``oracle.fugal_fp64.cugal``: scipy sparse products,
otherwise the reference's steps) on the Newman-Watts-Strogatz n=1000 workload
with the sparse path's semantics (and, after it, the dense path's), once with
the CUDA kernels' FP32 features and once with networkx's FP64 features, and
compares each mapping with the reference's own FP64 run stored in
``reference_nws1000.npz``.  The workload's nearly regular graph leaves many
rows with near-tied candidates, so rounding-level differences move rows to
other vertices; this measures that spread between FP64 implementations.
"""

import sys
import time
from pathlib import Path

import networkx as nx
import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def main():
    from cugal_b200.synthetic import make_pair
    from oracle import fugal_fp64 as O
    src, tgt, perm, _ = make_pair("nws1000")
    g = np.load(HERE / "reference_nws1000.npz")
    for variant, sparse in [("sparse", True), ("dense", False)]:
        for feats in ["cuda", "nx"]:
            t0 = time.time()
            p = O.OracleParams(sinkhorn_regularization=1e-3, sinkhorn_iterations=500, sinkhorn_threshold=1e-4,
                               sinkhorn_eval_freq=10, mu=1.0, iter_count=15, frank_wolfe_iter_count=10,
                               use_sparse_adjacency=sparse, double_lambda=True, hungarian_method="SCIPY")
            tr = O.FWTrace()
            _, mapping, _ = O.cugal(nx.Graph(src), nx.Graph(tgt), p, features=feats, trace=tr)
            cols = np.array([m[1] for m in mapping])
            print(f"{variant} path, {feats} features: accuracy {np.mean(cols == perm):.4f} (reference "
                  f"{float(g[variant + '_accuracy']):.4f}), same column as the reference "
                  f"{np.mean(cols == g[variant + '_cols']):.3f}, mean iterations {np.mean(tr.sinkhorn_iterations):.2f} "
                  f"(reference {g[variant + '_sk_iters'].mean():.2f}), {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()
