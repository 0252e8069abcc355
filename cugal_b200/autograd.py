"""Gradients through the log-domain Sinkhorn solve.

``sinkhorn_plan(C, config)`` is a ``torch.autograd.Function``: the forward runs
the device solve (``SinkhornState.solve``, reference ``cugal/sinkhorn.py:90-120``)
to convergence and returns the plan P = exp(-C/reg + u + v); the backward is the
implicit-function adjoint at the converged potentials, on the device:

    a = (G o P) 1,  b = (G o P)^T 1,   [I P; P^T I][alpha; beta] = [a; b]   (CG),
    dL/dC = -(1/reg) P o (G - alpha 1^T - 1 beta^T).

Each CG iteration is one pass over P (``fugal_plan_matvec`` forms P y and
P^T x together); the O(n) vector arithmetic runs in FP64.  The reference has no
backward pass; its torch ``solve_log`` differentiated by autograd is the check
(tests/test_gpu_adjoint.py), with central finite differences of the FP64 oracle.

``fw_objective`` is the Frank-Wolfe objective whose gradient the FW step uses
(cugal/pred.py:54-74): f(P) = -<P, A P B> + mu <D, P> + lam <P, 1 - P>, and
``tune_mu`` runs gradient steps on mu through the solve.
"""

from __future__ import annotations

import dataclasses

import torch

from . import _native as N
from .adjacency import Adjacency
from .config import Config, SinkhornMethod
from .sinkhorn import SinkhornState


class _Matvec:
    """Workspace-holding wrapper of fugal_plan_matvec for one n."""

    def __init__(self, n: int, device):
        self.n = n
        self.ws = torch.empty(N.workspace_size("fugal_plan_matvec_workspace_size", n), dtype=torch.uint8,
                              device=device)

    def __call__(self, P: torch.Tensor, x: torch.Tensor, y: torch.Tensor, W: torch.Tensor | None = None):
        """(P^T x, P y) with P optionally weighted elementwise by W."""
        Ptx = torch.empty(self.n, dtype=torch.float64, device=P.device)
        Py = torch.empty(self.n, dtype=torch.float64, device=P.device)
        N.call("fugal_plan_matvec", P.data_ptr(), N.matrix_ld(P, "P"), N.ptr(W),
               N.matrix_ld(W, "W") if W is not None else 0, self.n, x.data_ptr(), y.data_ptr(), Ptx.data_ptr(),
               Py.data_ptr(), self.ws.data_ptr(), self.ws.numel(), N.stream_handle(P.device))
        return Ptx, Py


def sinkhorn_adjoint(P: torch.Tensor, G: torch.Tensor, reg: float, tol: float = 1e-7, max_iter: int = 2000):
    """dL/dC for the converged plan P (n x n FP32 CUDA) and G = dL/dP; returns
    (dC FP32, CG iterations, final relative residual)."""
    N.require_cuda(P, "P", torch.float32)
    G = G.to(torch.float32).contiguous()
    n = P.shape[0]
    mv = _Matvec(n, P.device)
    ones = torch.ones(n, dtype=torch.float64, device=P.device)
    b, a = mv(P, ones, ones, W=G)          # b = (P o G)^T 1, a = (P o G) 1
    rhs = torch.cat([a, b])

    def apply(z):
        x, y = z[:n], z[n:]
        Ptx, Py = mv(P, x.contiguous(), y.contiguous())
        return torch.cat([x + Py, Ptx + y])

    z = torch.zeros(2 * n, dtype=torch.float64, device=P.device)
    r = rhs.clone()
    p = r.clone()
    rs = torch.dot(r, r)
    norm_rhs = torch.sqrt(rs).item()
    it, rel = 0, 0.0
    if norm_rhs > 0:
        for it in range(1, max_iter + 1):
            Ap = apply(p)
            alpha = rs / torch.dot(p, Ap)
            z += alpha * p
            r -= alpha * Ap
            rs_new = torch.dot(r, r)
            rel = torch.sqrt(rs_new).item() / norm_rhs
            if rel < tol:
                break
            p = r + (rs_new / rs) * p
            rs = rs_new
    alpha_v, beta_v = z[:n].contiguous(), z[n:].contiguous()
    dC = torch.empty((n, n), dtype=torch.float32, device=P.device)
    N.call("fugal_sinkhorn_adjoint", P.data_ptr(), N.matrix_ld(P, "P"), G.data_ptr(), N.matrix_ld(G, "G"), n,
           alpha_v.data_ptr(), beta_v.data_ptr(), -1.0 / reg, dC.data_ptr(), n, N.stream_handle(P.device))
    return dC, it, rel


class SinkhornPlan(torch.autograd.Function):
    """P = Sinkhorn(C) with the implicit adjoint as backward."""

    @staticmethod
    def forward(ctx, C, config, tol, max_iter):
        n = C.shape[0]
        state = SinkhornState(n, config)
        state.solve(C.detach().to(torch.float32).contiguous(), config)
        P = state.plan()
        ctx.save_for_backward(P)
        ctx.reg, ctx.tol, ctx.max_iter = config.sinkhorn_regularization, tol, max_iter
        return P

    @staticmethod
    def backward(ctx, G):
        (P,) = ctx.saved_tensors
        dC, _, _ = sinkhorn_adjoint(P, G, ctx.reg, ctx.tol, ctx.max_iter)
        return dC, None, None, None


def sinkhorn_plan(C: torch.Tensor, config: Config, tol: float = 1e-7, max_iter: int = 2000) -> torch.Tensor:
    """Differentiable converged plan of the log-domain solve on cost C (n x n CUDA)."""
    if config.sinkhorn_method != SinkhornMethod.LOG:
        raise NotImplementedError("the adjoint is implemented for SinkhornMethod.LOG")
    return SinkhornPlan.apply(C, dataclasses.replace(config, stream_dtype=None), tol, max_iter)


class SinkhornPlanUnrolled(torch.autograd.Function):
    """P after the reference's iteration (cugal/sinkhorn.py:108-115, no momentum)
    run from zero potentials, differentiated through the iterations: the duals
    are checkpointed every ``every`` iterations, each segment is recomputed on
    the way back, and every half step is reversed on the device
    (``fugal_sinkhorn_unrolled_step_backward``)."""

    @staticmethod
    def forward(ctx, C, config, every):
        n = C.shape[0]
        dev = C.device
        reg = config.sinkhorn_regularization
        K = (-C.detach().to(torch.float32) / reg).contiguous()
        Kt = K.t().contiguous()
        u = torch.zeros(n, dtype=torch.float32, device=dev)
        v = torch.zeros(n, dtype=torch.float32, device=dev)
        stream = N.stream_handle(dev)
        err = torch.zeros(1, dtype=torch.float64, device=dev)
        checkpoints = {0: (u.clone(), v.clone())}
        T = 0
        for t in range(config.sinkhorn_iterations):
            N.call("fugal_sinkhorn_log_step", Kt.data_ptr(), n, n, n, u.data_ptr(), v.data_ptr(), 1.0, stream)
            N.call("fugal_sinkhorn_log_step", K.data_ptr(), n, n, n, v.data_ptr(), u.data_ptr(), 1.0, stream)
            T = t + 1
            if T % every == 0:
                checkpoints[T] = (u.clone(), v.clone())
            if t % config.sinkhorn_eval_freq == 0 and t != 0:
                N.call("fugal_sinkhorn_log_marginal", K.data_ptr(), n, n, u.data_ptr(), v.data_ptr(), 0,
                       err.data_ptr(), stream)
                if err.item() < config.sinkhorn_threshold:
                    break
        P = torch.empty((n, n), dtype=torch.float32, device=dev)
        N.call("fugal_sinkhorn_plan", K.data_ptr(), n, n, u.data_ptr(), v.data_ptr(), P.data_ptr(), n, stream)
        ctx.save_for_backward(K, Kt, P)
        ctx.checkpoints, ctx.T, ctx.every, ctx.reg, ctx.uv = checkpoints, T, every, reg, (u, v)
        return P

    @staticmethod
    def backward(ctx, G):
        K, Kt, P = ctx.saved_tensors
        n = K.shape[0]
        dev = K.device
        stream = N.stream_handle(dev)
        mv = _Matvec(n, dev)
        ws = mv.ws
        ones = torch.ones(n, dtype=torch.float64, device=dev)
        G = G.to(torch.float32).contiguous()
        gK = (G * P).contiguous()
        gv, gu = mv(P, ones, ones, W=G)   # dL/dv_T = (G o P)^T 1, dL/du_T = (G o P) 1

        def step_back(out_dual, other_dual, g, axis, g_other):
            N.call("fugal_sinkhorn_unrolled_step_backward", K.data_ptr(), n, n, out_dual.data_ptr(),
                   other_dual.data_ptr(), g.data_ptr(), axis, gK.data_ptr(), n, g_other.data_ptr(), ws.data_ptr(),
                   ws.numel(), stream)

        T, every = ctx.T, ctx.every
        seg_end = T
        while seg_end > 0:
            seg_start = ((seg_end - 1) // every) * every
            u, v = (x.clone() for x in ctx.checkpoints[seg_start])
            states = [(u.clone(), v.clone())]          # (u_t, v_t) for t = seg_start .. seg_end
            for _ in range(seg_start, seg_end):
                N.call("fugal_sinkhorn_log_step", Kt.data_ptr(), n, n, n, u.data_ptr(), v.data_ptr(), 1.0, stream)
                N.call("fugal_sinkhorn_log_step", K.data_ptr(), n, n, n, v.data_ptr(), u.data_ptr(), 1.0, stream)
                states.append((u.clone(), v.clone()))
            for t in range(seg_end - 1, seg_start - 1, -1):
                u_t = states[t - seg_start][0]
                u_next, v_next = states[t + 1 - seg_start]
                # row half: u_{t+1} = -LSE_j(K + v_{t+1})
                step_back(u_next, v_next, gu, 1, gv)
                # column half: v_{t+1} = -LSE_i(K + u_t)
                gu = torch.zeros(n, dtype=torch.float64, device=dev)
                step_back(v_next, u_t, gv, 0, gu)
                gv = torch.zeros(n, dtype=torch.float64, device=dev)
            seg_end = seg_start
        return -gK / ctx.reg, None, None


def sinkhorn_plan_unrolled(C: torch.Tensor, config: Config, every: int = 10) -> torch.Tensor:
    """Differentiable plan of the reference's log-domain iteration, unrolled with
    dual checkpoints every ``every`` iterations (momentum not supported)."""
    if config.sinkhorn_method != SinkhornMethod.LOG or config.sinkhorn_momentum_start is not None:
        raise NotImplementedError("the unrolled adjoint covers SinkhornMethod.LOG without momentum")
    return SinkhornPlanUnrolled.apply(C.contiguous(), config, every)


def adjacency_product(A: Adjacency, M: torch.Tensor) -> torch.Tensor:
    """A @ M for a CSR adjacency and a dense FP32 matrix (device SpMM)."""
    return A.mul(M.contiguous())


def fw_objective(P: torch.Tensor, A: Adjacency, B: Adjacency, D: torch.Tensor, mu, lam: float = 0.0):
    """f(P) = -<P, A P B> + mu <D, P> + lam <P, 1 - P> (symmetric A, B): the
    objective whose gradient -2 A P B + mu D + lam (1 - 2P) the FW step uses."""
    APB = _APB.apply(P, A, B)
    return -(P * APB).sum() + mu * (D * P).sum() + lam * (P * (1 - P)).sum()


class _APB(torch.autograd.Function):
    """A P B for symmetric sparse A, B with its adjoint A G B."""

    @staticmethod
    def forward(ctx, P, A, B):
        ctx.A, ctx.B = A, B
        return adjacency_product(B, adjacency_product(A, P).t().contiguous()).t().contiguous()

    @staticmethod
    def backward(ctx, G):
        A, B = ctx.A, ctx.B
        return adjacency_product(B, adjacency_product(A, G.contiguous()).t().contiguous()).t().contiguous(), None, None


def structural_objective(P: torch.Tensor, A: Adjacency, B: Adjacency):
    """-<P, A P B>: the edge-agreement part of the objective (for a doubly
    stochastic P, ||A P - P B||^2 up to terms that do not depend on the match)."""
    return -(P * _APB.apply(P, A, B)).sum()


def tune_mu(A: Adjacency, B: Adjacency, D: torch.Tensor, config: Config, P0: torch.Tensor, mu0: float = 0.2,
            steps: int = 20, lr: float = 0.05, lam: float = 0.0):
    """Gradient descent on mu: C(mu) = -2 A P0 B + mu D + lam (1 - 2 P0), P(mu) =
    Sinkhorn(C(mu)) (converged plan, implicit adjoint), objective =
    structural_objective(P(mu)).  Each step moves along the normalised negative
    gradient with a backtracking (Armijo) line search that starts at twice the
    last accepted length (first: ``lr``), so the objective never increases.
    Returns one (mu, objective, d objective / d mu) per step."""
    base = (-2.0 * _APB.apply(P0, A, B) + lam * (1 - 2 * P0)).detach()

    def evaluate(mu_val: float, grad: bool):
        mu = torch.tensor(mu_val, dtype=torch.float64, device=P0.device, requires_grad=grad)
        C = base + mu.float() * D
        P = sinkhorn_plan(C, config)
        obj = structural_objective(P, A, B)
        if not grad:
            return float(obj.item()), 0.0
        (g,) = torch.autograd.grad(obj, mu)
        return float(obj.item()), float(g.item())

    mu_val = mu0
    obj, g = evaluate(mu_val, True)
    history = []
    length = lr
    for _ in range(steps):
        history.append((mu_val, obj, g))
        if g == 0.0:
            continue
        direction = -g / max(1.0, abs(g))
        t = length
        accepted = False
        for _ in range(10):
            cand = mu_val + t * direction
            obj_c, _ = evaluate(cand, False)
            if obj_c <= obj + 1e-4 * t * g * direction:
                accepted = True
                break
            t *= 0.5
        if not accepted:
            continue  # no decrease along the gradient at this resolution: stay
        mu_val = cand
        obj, g = evaluate(mu_val, True)
        length = 2.0 * t
    return history
