"""Exact rounding on the device (the reference's ``HungarianMethod.SCIPY``,
``cugal/pred.py:151-158``): the same mapping as
``scipy.optimize.linear_sum_assignment(P, maximize=True)``, computed by
``fugal_exact_lap`` without copying P to the host."""

from __future__ import annotations

import torch

from . import _native as N

FUGAL_OK, FUGAL_ITER_LIMIT = 0, 4


def default_max_steps(n: int) -> int:
    """Cap on Dijkstra steps: n per row, a bound no shortest-augmenting-path run
    exceeds (each step of a row's search settles one more column), so reaching it
    means a fault, not a hard instance.  A converged Frank-Wolfe P needs about one
    step per row."""
    return n * n + 1024


def exact_assign(P: torch.Tensor, maximize: bool = True, max_steps: int | None = None):
    """(columns int64 device tensor, steps int64 device tensor, status int32 device
    tensor) for a square FP32 CUDA matrix P.  Asynchronous: read ``status`` before
    using ``columns`` (FUGAL_OK = 0)."""
    N.require_cuda(P, "P", torch.float32)
    n = P.shape[0]
    if P.dim() != 2 or P.shape[1] != n:
        raise ValueError("exact_assign: P must be square")
    ldp = N.matrix_ld(P, "P")
    cols = torch.empty(n, dtype=torch.int64, device=P.device)
    steps = torch.zeros(1, dtype=torch.int64, device=P.device)
    status = torch.full((1,), -1, dtype=torch.int32, device=P.device)
    ws = torch.empty(N.workspace_size("fugal_exact_lap_workspace_size", n), dtype=torch.uint8, device=P.device)
    N.call("fugal_exact_lap", P.data_ptr(), ldp, n, int(maximize), int(max_steps or default_max_steps(n)),
           cols.data_ptr(), steps.data_ptr(), status.data_ptr(), ws.data_ptr(), ws.numel(),
           N.stream_handle(P.device))
    return cols, steps, status
