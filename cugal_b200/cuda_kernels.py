"""Drop-in replacement of cuGAL's pybind11 module ``cuda_kernels``.

Same function names, argument order and in-place semantics as
``cuda_kernels/kernels.cpp:32-70``, implemented on ``libfugal_b200.so``:
outputs are caller-allocated CUDA tensors written in place; the two functions
that return a float (the reference synchronises the device inside them) read
the FP64 device result back.  Launches go to torch's current stream instead of
the legacy default stream, and no call ends in a device-wide synchronize.
"""

from __future__ import annotations

import torch

from . import _native as N
from .greedy_lap import greedy_assign
from .config import HungarianMethod


def _ld(t: torch.Tensor, name: str) -> int:
    return N.matrix_ld(t, name)


def adjacency_matmul(col_indices, row_pointers, matrix, out, negate_lhs: bool) -> None:
    """out = (+-A) @ matrix (``kernels.cpp:33-36``).  A non-contiguous ``matrix`` is
    taken as the transpose of a contiguous one and ``out`` must then have the
    same (transposed) strides, as ``torch.empty_like(matrix)`` gives."""
    n = row_pointers.numel() - 1
    stream = N.stream_handle(matrix.device)
    if matrix.is_contiguous():
        N.call("fugal_adjacency_matmul", col_indices.data_ptr(), row_pointers.data_ptr(), n, matrix.data_ptr(),
               _ld(matrix, "matrix"), 0, out.data_ptr(), _ld(out, "out"), int(negate_lhs), stream)
    else:
        q, o = matrix.t(), out.t()
        N.call("fugal_adjacency_matmul", col_indices.data_ptr(), row_pointers.data_ptr(), n, q.data_ptr(),
               _ld(q, "matrix^T"), 1, o.data_ptr(), _ld(o, "out^T"), int(negate_lhs), stream)


def create_adjacency(edges, col_indices, row_pointers) -> None:
    """CSR from a flat int32 edge list [x0, y0, x1, y1, ...] (``kernels.cpp:37-39``)."""
    m = edges.numel() // 2
    n = row_pointers.numel() - 1
    ws = torch.empty(N.workspace_size("fugal_create_adjacency_workspace_size", m, n), dtype=torch.uint8,
                     device=edges.device)
    N.call("fugal_create_adjacency", edges.data_ptr(), m, n, col_indices.data_ptr(), row_pointers.data_ptr(),
           ws.data_ptr(), ws.numel(), N.stream_handle(edges.device))


def graph_features(col_indices, row_pointers, clustering, degrees) -> None:
    """Degree and clustering coefficient per vertex (``kernels.cpp:42``)."""
    n = row_pointers.numel() - 1
    N.call("fugal_graph_features", col_indices.data_ptr(), row_pointers.data_ptr(), n, clustering.data_ptr(),
           degrees.data_ptr(), None, None, N.stream_handle(clustering.device))


def average_neighbor_features(col_indices, row_pointers, features, averages) -> None:
    """Mean of a vertex feature over each vertex's neighbours (``kernels.cpp:43-46``)."""
    n = row_pointers.numel() - 1
    N.call("fugal_average_neighbor_features", col_indices.data_ptr(), row_pointers.data_ptr(), n,
           features.data_ptr(), averages.data_ptr(), N.stream_handle(features.device))


def sinkhorn_log_step(K, add, out, momentum: float) -> None:
    """out = (1-w) out - w LSE_rows(K + add) (``kernels.cpp:49-52``)."""
    N.call("fugal_sinkhorn_log_step", K.data_ptr(), K.shape[0], K.shape[1], _ld(K, "K"), add.data_ptr(),
           out.data_ptr(), float(momentum), N.stream_handle(K.device))


def sinkhorn_log_marginal(K, u, v) -> float:
    """Row-marginal L1 error as the reference kernel computes it (``kernels.cpp:53-56``)."""
    res = torch.zeros(1, dtype=torch.float64, device=K.device)
    N.call("fugal_sinkhorn_log_marginal", K.data_ptr(), K.shape[0], _ld(K, "K"), u.data_ptr(), v.data_ptr(), 1,
           res.data_ptr(), N.stream_handle(K.device))
    return float(res.item())


def add_distance(source, target, out) -> None:
    """out += euclidean distance of the 4-feature rows (``kernels.cpp:59``)."""
    N.call("fugal_add_distance", source.data_ptr(), target.data_ptr(), out.shape[0], out.data_ptr(),
           _ld(out, "out"), N.stream_handle(out.device))


def regularize(gradient, P, iteration: int) -> None:
    """gradient += iteration - 2 iteration P (``kernels.cpp:62``)."""
    N.call("fugal_regularize", gradient.data_ptr(), _ld(gradient, "gradient"), P.data_ptr(), _ld(P, "P"),
           gradient.shape[0], int(iteration), N.stream_handle(gradient.device))


def update_quasi_permutation_log(P, K, u, v, alpha: float, regularization: float) -> float:
    """P += alpha (exp(K+u+v) - P); returns |duality gap| (``kernels.cpp:65``)."""
    gap = torch.zeros(1, dtype=torch.float64, device=P.device)
    N.call("fugal_update_quasi_permutation_log", P.data_ptr(), _ld(P, "P"), K.data_ptr(), _ld(K, "K"),
           u.data_ptr(), v.data_ptr(), P.shape[0], float(alpha), float(regularization), gap.data_ptr(),
           N.stream_handle(P.device))
    return abs(float(gap.item()))


def dense_hungarian(cost, out) -> None:
    """The reference binds a GPU Munkres here (``kernels.cpp:68``) that cugal never
    calls; this library offers the greedy rounding kernels instead."""
    raise NotImplementedError("dense_hungarian is not provided; use cugal_b200.greedy_lap or SCIPY")
