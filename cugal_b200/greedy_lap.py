"""Greedy rounding (reference ``cugal/greedy_lap.py:7-85``) on the GPU.

Same result as the reference for GREEDY, DOUBLE_GREEDY, PARALLEL_GREEDY and
RAND given the same P (and, for RAND, the same ``torch.randperm`` draw), with
P mutated the way the reference mutates it.  Rows whose maxima tie are ordered
by row index (the reference's ``argsort`` is unstable there).  MORE_RAND draws
its row order with ``torch.randperm`` and one ``random.random()`` per row, as
the reference does, and samples each row's column on the device
(``fugal_sampled_lap``); its running sums are FP64 (the reference's are in P's
dtype), so a draw that lands within rounding of a column boundary may pick the
neighbouring column.
"""

from __future__ import annotations

import random

import torch

from . import _native as N
from .config import Config, HungarianMethod

_METHODS = {
    HungarianMethod.GREEDY: N.LAP_GREEDY,
    HungarianMethod.DOUBLE_GREEDY: N.LAP_DOUBLE_GREEDY,
    HungarianMethod.PARALLEL_GREEDY: N.LAP_PARALLEL_GREEDY,
    HungarianMethod.RAND: N.LAP_ORDERED,
}


def sampled_assign(P: torch.Tensor, order: torch.Tensor | None = None, uniforms=None,
                   mutate: bool = True) -> torch.Tensor:
    """MORE_RAND rounding (``cugal/greedy_lap.py:34-48``): column per row (int64
    device tensor).  ``order`` defaults to ``torch.randperm(n)`` on P's device and
    ``uniforms`` to n draws of ``random.random()``, the reference's draws."""
    N.require_cuda(P, "P", torch.float32)
    n = P.shape[0]
    ldp = N.matrix_ld(P, "P")
    if order is None:
        order = torch.randperm(n, device=P.device)
    order = torch.as_tensor(order).to(device=P.device, dtype=torch.int64).contiguous()
    if uniforms is None:
        uniforms = [random.random() for _ in range(n)]
    u = torch.as_tensor(uniforms, dtype=torch.float64).to(P.device).contiguous()
    cols = torch.empty(n, dtype=torch.int64, device=P.device)
    N.call("fugal_sampled_lap", P.data_ptr(), ldp, n, order.data_ptr(), u.data_ptr(), int(mutate), cols.data_ptr(),
           N.stream_handle(P.device))
    return cols


def greedy_assign(P: torch.Tensor, method: HungarianMethod, candidates: int = 8, mutate: bool = True,
                  order: torch.Tensor | None = None) -> torch.Tensor:
    """Column per row (int64 device tensor) for a square FP32 CUDA matrix P."""
    if method == HungarianMethod.MORE_RAND:
        return sampled_assign(P, order, mutate=mutate)
    if method not in _METHODS:
        raise NotImplementedError(f"{method} is not available on the GPU path")
    N.require_cuda(P, "P", torch.float32)
    n = P.shape[0]
    ldp = N.matrix_ld(P, "P")
    if method == HungarianMethod.RAND:
        if order is None:
            order = torch.randperm(n, device=P.device)
        order = order.to(device=P.device, dtype=torch.int64).contiguous()
    cols = torch.empty(n, dtype=torch.int64, device=P.device)
    ws = torch.empty(N.workspace_size("fugal_greedy_lap_workspace_size", n, candidates), dtype=torch.uint8,
                     device=P.device)
    N.call("fugal_greedy_lap", P.data_ptr(), ldp, n, _METHODS[method], N.ptr(order), candidates, int(mutate),
           cols.data_ptr(), ws.data_ptr(), ws.numel(), N.stream_handle(P.device))
    return cols


def greedy_lap(cost_matrix: torch.Tensor, config: Config) -> list:
    """``greedy_lap`` (``cugal/greedy_lap.py:7``): list of column indices."""
    cols = greedy_assign(cost_matrix, config.hungarian_method, config.lap_candidates)
    return cols.cpu().tolist()
