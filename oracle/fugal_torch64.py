"""FP64 restatement of the FUGAL Frank-Wolfe loop in torch, for large n on a GPU.

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never part of it.

The same algorithm as ``oracle/fugal_fp64.py`` (which is pinned to the
reference's own outputs by ``tests/test_oracle_golden.py``), written with torch
tensors so that the FP64 computation runs on a GPU at sizes the numpy oracle
cannot reach (n = 32768: 8.6 GB per FP64 matrix).  ``tests/test_oracle_torch64.py``
checks it against the numpy oracle on the CPU.  Reference lines restated:

* gradient  -2 A P B + D + lam (1 - 2P)  (``cugal/pred.py:54-74``; dense
  semantics with the doubled lambda term, ``cugal/pred.py:38-51``);
* log-domain Sinkhorn ``SinkhornState.solve_log`` (``cugal/sinkhorn.py:90-120``)
  with the non-mutating column-marginal error (``cugal/sinkhorn.py:76``), warm
  started across solves, no momentum unless ``momentum_start`` is given
  (``cugal/sinkhorn.py:78-88``);
* the update P += alpha (q - P), alpha = 2 / (2 + it), and the duality gap
  |sum G (q - P)| (``cugal/pred.py:77-86,133-141``);
* the Frank-Wolfe schedule of ``find_quasi_permutation_matrix``
  (``cugal/pred.py:89-148``);
* DOUBLE_GREEDY rounding (``cugal/greedy_lap.py:50-63``).

The n x n temporaries of the row and column log-sum-exps are formed a block of
rows at a time, so the memory held is P, K and one block.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch


def csr_tensor(row_pointers, col_indices, n: int, device, dtype=torch.float64) -> torch.Tensor:
    """Sparse CSR adjacency (values 1) from CSR arrays."""
    rp = torch.as_tensor(np.asarray(row_pointers, dtype=np.int64), device=device)
    ci = torch.as_tensor(np.asarray(col_indices, dtype=np.int64), device=device)
    vals = torch.ones(ci.numel(), dtype=dtype, device=device)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)  # "sparse CSR support is in beta"
        return torch.sparse_csr_tensor(rp, ci, vals, size=(n, n), check_invariants=True)


def distance_into(out: torch.Tensor, F1: torch.Tensor, F2: torch.Tensor, block: int) -> None:
    """out += ||F1_i - F2_j|| by direct differences (``cugal/feature_extraction.py:106-108``)."""
    n = out.shape[0]
    for r0 in range(0, n, block):
        d = F1[r0:r0 + block, None, :] - F2[None, :, :]
        out[r0:r0 + block] += torch.sqrt(torch.sum(d * d, dim=-1))


def sparse_gradient_into(G: torch.Tensor, A: torch.Tensor, B: torch.Tensor, P: torch.Tensor, F1, F2,
                         lam: float, lam_scale: float, block: int) -> None:
    """G = -2 A P B + D + c lam (1 - 2P) for symmetric A, B (``cugal/pred.py:54-74``;
    c = 2 restates the dense path's doubled term, ``cugal/pred.py:45-50``)."""
    AP = A @ P
    APt = AP.t().contiguous()
    del AP
    BAPt = B @ APt
    del APt
    G.copy_(BAPt.t())
    del BAPt
    G.mul_(-2.0)
    distance_into(G, F1, F2, block)
    if lam != 0.0:
        for _ in range(int(lam_scale)):
            G.add_(lam - lam * 2.0 * P)


def _column_lse(K: torch.Tensor, u: torch.Tensor, block: int) -> torch.Tensor:
    """LSE over i of K[i, j] + u[i] (torch.logsumexp semantics), a block of rows at a time."""
    n = K.shape[0]
    m = torch.full((K.shape[1],), -torch.inf, dtype=K.dtype, device=K.device)
    parts = []
    for r0 in range(0, n, block):
        x = K[r0:r0 + block] + u[r0:r0 + block, None]
        bm = torch.amax(x, dim=0)
        parts.append((r0, bm))
        m = torch.maximum(m, bm)
    m_safe = torch.where(torch.isfinite(m), m, torch.zeros_like(m))
    s = torch.zeros_like(m)
    for r0, _ in parts:
        x = K[r0:r0 + block] + u[r0:r0 + block, None]
        s += torch.sum(torch.exp(x - m_safe[None, :]), dim=0)
    return torch.log(s) + m_safe


def _row_lse(K: torch.Tensor, v: torch.Tensor, block: int) -> torch.Tensor:
    n = K.shape[0]
    out = torch.empty(n, dtype=K.dtype, device=K.device)
    for r0 in range(0, n, block):
        out[r0:r0 + block] = torch.logsumexp(K[r0:r0 + block] + v[None, :], dim=1)
    return out


def marginal_error(K: torch.Tensor, u: torch.Tensor, v: torch.Tensor, block: int) -> float:
    """sum_j |sum_i exp(K + u + v) - 1| (``cugal/sinkhorn.py:76``)."""
    cs = torch.zeros(K.shape[1], dtype=K.dtype, device=K.device)
    for r0 in range(0, K.shape[0], block):
        cs += torch.sum(torch.exp(K[r0:r0 + block] + u[r0:r0 + block, None] + v[None, :]), dim=0)
    return float(torch.sum(torch.abs(cs - 1.0)).item())


def lehmann_momentum(errors, momentum_start, eval_freq: int) -> float:
    """``SinkhornState.lehmann_momentum`` (``cugal/sinkhorn.py:78-88``)."""
    import math
    if momentum_start is None or len(errors) * eval_freq < momentum_start:
        return 1.0
    index = momentum_start // eval_freq
    if len(errors) < index - 1:
        return 1.0
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.float64(errors[index - 1]) / np.float64(errors[index - 2])
    ratio = min(float(ratio), 0.99)
    if math.isnan(ratio):
        ratio = 0.99
    return 2.0 / (1.0 + math.sqrt(1 - ratio ** (1.0 / eval_freq)))


@dataclass
class SolveRecord:
    iterations: int
    errors: list


def sinkhorn_log_solve_(K: torch.Tensor, u: torch.Tensor, v: torch.Tensor, max_iter: int, threshold: float,
                        eval_freq: int, momentum_start=None, block: int = 1024) -> SolveRecord:
    """``SinkhornState.solve_log`` (``cugal/sinkhorn.py:90-120``) on K = -C / reg;
    u, v are the warm start and are updated in place."""
    errors: list[float] = []
    momentum = 1.0
    it = 0
    for it in range(max_iter):
        v.copy_(v * (1 - momentum) - momentum * _column_lse(K, u, block))
        u.copy_(u * (1 - momentum) - momentum * _row_lse(K, v, block))
        if it % eval_freq == 0 and it != 0:
            errors.append(marginal_error(K, u, v, block))
            if errors[-1] < threshold:
                break
            momentum = lehmann_momentum(errors, momentum_start, eval_freq)
    return SolveRecord(it + 1, errors)


def update_(P: torch.Tensor, K: torch.Tensor, u: torch.Tensor, v: torch.Tensor, alpha: float, reg: float,
            block: int) -> float:
    """P += alpha (q - P), q = exp(K + u + v); returns |sum G (q - P)| with G = -reg K
    (``cugal/pred.py:77-86,139-141``)."""
    gap = 0.0
    for r0 in range(0, P.shape[0], block):
        q = torch.exp(K[r0:r0 + block] + u[r0:r0 + block, None] + v[None, :])
        d = q - P[r0:r0 + block]
        gap += float(torch.sum((-reg * K[r0:r0 + block]) * d).item())
        P[r0:r0 + block] += alpha * d
    return abs(gap)


@dataclass
class Trace:
    sinkhorn_iterations: list = field(default_factory=list)
    sinkhorn_final_errors: list = field(default_factory=list)
    gaps: list = field(default_factory=list)
    objectives: list = field(default_factory=list)


def objective(A: torch.Tensor, B: torch.Tensor, P: torch.Tensor, F1, F2, lam_eff: float, block: int) -> dict:
    """-<P, A P B> + <D, P> + lam_eff <P, 1 - P> and its terms, FP64."""
    AP = A @ P
    APt = AP.t().contiguous()
    del AP
    BAPt = B @ APt
    del APt
    structural = float(torch.sum(P * BAPt.t()).item())
    del BAPt
    feature = 0.0
    for r0 in range(0, P.shape[0], block):
        d = F1[r0:r0 + block, None, :] - F2[None, :, :]
        feature += float(torch.sum(torch.sqrt(torch.sum(d * d, dim=-1)) * P[r0:r0 + block]).item())
    concave = float(torch.sum(P * (1.0 - P)).item())
    return {"structural": structural, "feature": feature, "concave": concave,
            "objective": -structural + feature + lam_eff * concave}


def find_quasi_permutation_matrix(A_csr, B_csr, F1: np.ndarray, F2: np.ndarray, *, reg: float, iter_count: int,
                                  fw_iter_count: int, sinkhorn_iterations: int, threshold: float,
                                  eval_freq: int, mu: float = 1.0, lam_scale: float = 1.0, device="cuda",
                                  block: int = 1024, max_steps: int | None = None,
                                  trace: Trace | None = None, objective_every: bool = False) -> torch.Tensor:
    """``find_quasi_permutation_matrix`` (``cugal/pred.py:89-148``) in FP64 on
    ``device``; ``max_steps`` stops after that many Frank-Wolfe steps (a truncated
    run).  F1, F2: the unscaled n x 4 feature matrices (scaled by mu here)."""
    n = F1.shape[0]
    A = csr_tensor(*A_csr, n, device)
    B = csr_tensor(*B_csr, n, device)
    f1 = torch.as_tensor(np.asarray(F1, dtype=np.float64) * mu, device=device)
    f2 = torch.as_tensor(np.asarray(F2, dtype=np.float64) * mu, device=device)
    P = torch.full((n, n), 1.0 / n, dtype=torch.float64, device=device)
    K = torch.empty_like(P)
    u = torch.zeros(n, dtype=torch.float64, device=device)
    v = torch.zeros(n, dtype=torch.float64, device=device)
    steps = 0
    for lam in range(iter_count):
        for it in range(1, fw_iter_count + 1):
            if max_steps is not None and steps >= max_steps:
                return P
            sparse_gradient_into(K, A, B, P, f1, f2, float(lam), lam_scale, block)
            K.mul_(-1.0 / reg)
            rec = sinkhorn_log_solve_(K, u, v, sinkhorn_iterations, threshold, eval_freq, block=block)
            gap = update_(P, K, u, v, 2.0 / (2.0 + it), reg, block)
            steps += 1
            if trace is not None:
                trace.sinkhorn_iterations.append(rec.iterations)
                trace.sinkhorn_final_errors.append(rec.errors[-1] if rec.errors else float("nan"))
                trace.gaps.append(gap)
                if objective_every:
                    trace.objectives.append(objective(A, B, P, f1, f2, lam * lam_scale, block)["objective"])
    return P


def double_greedy(P: torch.Tensor) -> np.ndarray:
    """DOUBLE_GREEDY rounding (``cugal/greedy_lap.py:50-63``) on a copy of P, rows
    ordered by descending row maximum (ties by row index)."""
    Q = P.clone()
    n = Q.shape[0]
    order = torch.argsort(-Q.max(dim=1).values, stable=True).cpu().numpy()
    taken = torch.ones(n, dtype=Q.dtype, device=Q.device)
    res = np.zeros(n, dtype=np.int64)
    for r in order:
        Q[r] *= taken
        m = int(torch.argmax(Q[r]).item())
        taken[m] = 0
        res[r] = m
    return res


def solve_log_differentiable(C: torch.Tensor, reg: float, iterations: int, segment: int = 25) -> torch.Tensor:
    """The reference's ``solve_log`` (``cugal/sinkhorn.py:99-116``, no momentum,
    zero start) as plain differentiable torch ops for ``iterations`` iterations:
    K = -C/reg; v = -LSE_i(K + u), u = -LSE_j(K + v); returns P = exp(K + u + v).
    Autograd through it is torch autograd through the reference's iteration;
    the iterations are recomputed segment by segment on the way back
    (``torch.utils.checkpoint``) so the memory held is one segment's."""
    import torch.utils.checkpoint as ckpt
    K = -C / reg
    n = C.shape[0]
    u = torch.zeros(n, dtype=C.dtype, device=C.device)
    v = torch.zeros(n, dtype=C.dtype, device=C.device)

    def run(K, u, v, k):
        for _ in range(k):
            v = -torch.logsumexp(K + u[:, None], dim=0)
            u = -torch.logsumexp(K + v[None, :], dim=1)
        return u, v

    done = 0
    while done < iterations:
        k = min(segment, iterations - done)
        u, v = ckpt.checkpoint(run, K, u, v, k, use_reentrant=False)
        done += k
    return torch.exp(K + u[:, None] + v[None, :])
