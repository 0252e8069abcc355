"""Golden gradients of the reference's log-domain Sinkhorn under torch autograd.

Runs the reference's own SinkhornState.solve_log (cugal/sinkhorn.py:90-120) on
the CPU in FP64 with autograd enabled, the convergence check replaced by its
non-mutating form (as in make_golden.py), forms P = exp(K + u + v) and
L = sum(W o P), and records dL/dC.  Output: reference_adjoint.npz next to this
script.  Run where the reference is checked out:
    python tests/golden/make_adjoint_golden.py
"""

import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import import_reference, patched_marginal_error_log  # noqa: E402


def main():
    cugal = import_reference()
    from cugal.config import Config, SinkhornMethod
    from cugal.sinkhorn import SinkhornState
    SinkhornState.marginal_error_log = patched_marginal_error_log
    out = {}
    for k, (n, reg, iters) in enumerate([(16, 0.5, 400), (24, 0.3, 600)]):
        rng = np.random.default_rng(100 + k)
        C0 = rng.random((n, n)) * 3.0
        W = rng.standard_normal((n, n))
        cfg = Config(device="cpu", dtype=torch.float64, sinkhorn_method=SinkhornMethod.LOG,
                     sinkhorn_regularization=reg, sinkhorn_iterations=iters, sinkhorn_threshold=1e-13,
                     sinkhorn_eval_freq=10)
        C = torch.tensor(C0, dtype=torch.float64, requires_grad=True)
        state = SinkhornState(n, cfg)
        K, u, v = state.solve(C, cfg)
        P = torch.exp(K + u[:, None] + v[None, :])
        L = (torch.tensor(W) * P).sum()
        L.backward()
        out[f"C{k}"] = C0
        out[f"W{k}"] = W
        out[f"reg{k}"] = np.array(reg)
        out[f"P{k}"] = P.detach().numpy()
        out[f"dC{k}"] = C.grad.numpy()
    np.savez(HERE / "reference_adjoint.npz", **out)


if __name__ == "__main__":
    main()
