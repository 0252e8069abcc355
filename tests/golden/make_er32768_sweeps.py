"""Per-solve Sinkhorn iteration counts of the FP64 restatement of the reference on
the Erdos-Renyi n=32768 workload (mean degree 16, seed 2, 2% noise; mu 1,
15 x 10 Frank-Wolfe steps, log Sinkhorn reg 1e-3, at most 500 iterations,
tolerance 1e-4 checked every 10, non-mutating marginal check).

    python tests/golden/make_er32768_sweeps.py [out.json]     # needs a CUDA device (FP64 on the GPU)

The counts are what the reference's CPU FP64 path (with its marginal check made
non-mutating) would run on this workload; bench.py scales its CPU per-iteration
timing by them.  Default output: tests/golden/er32768_fp64_sweeps.json.
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def main():
    from cugal_b200.synthetic import make_pair
    from oracle import fugal_fp64 as O
    from oracle import fugal_torch64 as T
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "er32768_fp64_sweeps.json"
    src, tgt, perm, w = make_pair("er32768")
    A_csr, B_csr = O.csr_from_graph(src), O.csr_from_graph(tgt)
    F1 = O.features_cuda_semantics(*A_csr).astype(np.float64)
    F2 = O.features_cuda_semantics(*B_csr).astype(np.float64)
    trace = T.Trace()
    t0 = time.perf_counter()
    P = T.find_quasi_permutation_matrix(A_csr, B_csr, F1, F2, reg=1e-3, iter_count=15, fw_iter_count=10,
                                        sinkhorn_iterations=500, threshold=1e-4, eval_freq=10, mu=1.0,
                                        device="cuda", block=1024, trace=trace)
    secs = time.perf_counter() - t0
    cols = T.double_greedy(P)
    rec = {"workload": w.name, "n": int(src.number_of_nodes()),
           "sinkhorn_iterations": [int(x) for x in trace.sinkhorn_iterations],
           "final_errors": [float(x) for x in trace.sinkhorn_final_errors],
           "node_accuracy_double_greedy": float(np.mean(cols == perm)), "seconds": secs,
           "generator": "tests/golden/make_er32768_sweeps.py (oracle/fugal_torch64.py, FP64 on the GPU)"}
    out.write_text(json.dumps(rec, indent=1))
    print(f"wrote {out}: mean {np.mean(rec['sinkhorn_iterations']):.2f} iterations per solve, "
          f"{sum(1 for x in rec['sinkhorn_iterations'] if x >= 500)} capped, accuracy "
          f"{rec['node_accuracy_double_greedy']:.4f}, {secs:.0f} s")


if __name__ == "__main__":
    main()
