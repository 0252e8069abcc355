"""The reference's FP32 GPU path on its own compiled kernels (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Loads the reference's ``cuda_kernels`` extension
built by ``oracle/build_ref.py`` and restates, line for line in behaviour, the
Python that drives it on CUDA:

* ``sparse_gradient``  -- cugal/pred.py:54-74 (B.mul(A.mul(P).T).T * -2, then
  add_distance or += D, then regularize);
* ``solve_log``        -- cugal/sinkhorn.py:90-120 GPU branch (K = -C/reg, a
  transposed copy, two sinkhorn_log_step launches per iteration, the
  marginal check every eval_freq iterations).  ``mutating_marginal`` selects
  the reference's in-place method (Q1) or the non-mutating form;
* ``update``           -- update_quasi_permutation_log (cugal/pred.py:134-136).

Used to cross-check the B200 kernels against the reference's kernels on
identical inputs and to time the reference GPU path.  The reference's kernels
launch on the legacy default stream and synchronise the device themselves.
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
from pathlib import Path

import torch

REF_SO = Path(__file__).resolve().parent / "_ref" / "cuda_kernels.so"


def available() -> bool:
    return REF_SO.exists()


_mod = None


def kernels():
    global _mod
    if _mod is None:
        loader = importlib.machinery.ExtensionFileLoader("cuda_kernels", str(REF_SO))
        spec = importlib.util.spec_from_file_location("cuda_kernels", str(REF_SO), loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _mod = mod
    return _mod


def adjacency_mul(col, rp, M, negate=False):
    """Adjacency.mul (cugal/adjacency.py:128-156) on the reference kernel."""
    out = torch.empty_like(M)
    kernels().adjacency_matmul(col, rp, M, out, negate)
    return out


def sparse_gradient(A, B, P, features, lam: int):
    """A, B: (col, rp) pairs; features: (source, target) rows or a D matrix."""
    ck = kernels()
    G = adjacency_mul(*B, adjacency_mul(*A, P).T).T
    G *= -2
    if isinstance(features, tuple):
        ck.add_distance(features[0], features[1], G)
    else:
        G += features
    ck.regularize(G, P, lam)
    return G


def marginal_error(K, u, v, mutate: bool) -> float:
    if mutate:  # cugal/sinkhorn.py:67-74
        K += u[:, None]
        K += v[None, :]
        torch.exp(K, out=K)
        K -= u[:, None]
        K -= v[None, :]
        return torch.sum(abs(torch.sum(K, dim=0) - 1)).item()
    return torch.sum(abs(torch.sum(torch.exp(K + u[:, None] + v[None, :]), dim=0) - 1)).item()


def lehmann(errors, momentum_start, eval_freq):
    from oracle.fugal_fp64 import lehmann_momentum
    return lehmann_momentum(errors, momentum_start, eval_freq)


def solve_log(C, u, v, reg, max_iter, threshold, eval_freq, momentum_start=None, mutating_marginal=False):
    """Returns (K, u, v, iteration_count, errors); u, v updated in place like the reference."""
    ck = kernels()
    K = -C / reg
    K_t = K.t().contiguous()
    errors, momentum = [], 1.0
    iteration = 0
    for iteration in range(max_iter):
        ck.sinkhorn_log_step(K_t, u, v, momentum)
        ck.sinkhorn_log_step(K, v, u, momentum)
        if iteration % eval_freq == 0 and iteration != 0:
            errors.append(marginal_error(K, u, v, mutating_marginal))
            if errors[-1] < threshold:
                break
            momentum = lehmann(errors, momentum_start, eval_freq)
    return K, u, v, iteration + 1, errors


def update(P, K, u, v, alpha, reg) -> float:
    return kernels().update_quasi_permutation_log(P, K, u, v, alpha, reg)
